"""The batched engine on a B200 (-m gpu): results identical alone, in a mix,
with and without graph replay, and to the single-search engine; every hit
re-derived by the oracle; the first hits really are the first."""
import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import batch as B
from onion_gen_b200 import run, workloads

pytestmark = pytest.mark.gpu

SEARCHES = [
    (101, ["ab", "cd"], 5),
    (102, ["xyz"], 3),
    (103, [workloads.SplitMix64(77 + i).prefix(4, 4) for i in range(200)], 8),
    (104, ["q7", "lmn", "uvwx"], 4),
    (105, ["k2"], 16),
    (106, [workloads.SplitMix64(9).prefix(5, 5)], 1),
]
SMALL = dict(half=64, slots=128 * 64)


def key_of(h):
    return (h.offset, h.packed)


def run_batch(device, searches, **kw):
    b = B.Batch(device, **{**SMALL, **kw})
    for sid, prefixes, quota in searches:
        b.admit(sid, workloads.seed(sid), prefixes, quota)
    steps = 0
    while b.running():
        b.step()
        steps += 1
        assert steps < 5000
    out = {sid: [key_of(h) for h in b.results(sid)] for sid, _, _ in searches}
    for sid, _, quota in searches:
        st = b.status(sid)
        assert st.done == 1 and st.hits == quota
    b.close()
    return out, steps


@pytest.fixture(scope="module")
def mixed(device):
    return run_batch(device, SEARCHES)


def test_mixed_equals_alone(device, mixed):
    out, steps = mixed
    assert steps > 1
    for s in SEARCHES:
        alone, _ = run_batch(device, [s])
        assert alone[s[0]] == out[s[0]], s[0]


def test_graph_and_plain_launches_agree(device, mixed):
    out, _ = mixed
    plain, _ = run_batch(device, SEARCHES, graph=False)
    assert plain == out


def test_other_shapes_agree(device, mixed):
    """Lane count, rounds per step and pool size change how much is examined,
    never which hits come first."""
    out, _ = mixed
    other, _ = run_batch(device, SEARCHES, slots=128 * 23, rounds=3)
    assert other == out


def test_single_engine_agrees(device, mixed):
    out, _ = mixed
    for sid, prefixes, quota in SEARCHES:
        cfg = N.EngineConfig(0, 64, 1024, 2, 128, 0, 0)
        found, _, _ = run.device_search(device, workloads.seed(sid), prefixes, quota, config=cfg)
        assert [(h.offset, h.packed) for h in found] == out[sid], sid


def test_every_hit_rederives_in_the_oracle(device, oracle, mixed):
    out, _ = mixed
    for sid, prefixes, quota in SEARCHES:
        seed = workloads.seed(sid)
        fs = oracle.FilterSet(prefixes)
        for off, packed in out[sid]:
            sec = oracle.expanded_secret_at_offset(seed, off)
            pk = oracle.pack(oracle.scalar_base_mult(sec[:32]))
            assert pk[:31] == packed[:31] and pk[31] & 0x7F == packed[31]
            assert fs.match(packed) >= 0


def test_first_hits_are_the_first(device, oracle, mixed):
    """An oracle scan of the first candidates finds exactly the same first
    hits (offsets start at 8 and every multiple of 8 is examined)."""
    out, _ = mixed
    for sid, prefixes, quota in SEARCHES[:2] + SEARCHES[3:5]:
        seed = workloads.seed(sid)
        start = oracle.scalar_base_mult(oracle.secret_scalar(seed))
        fs = oracle.FilterSet(prefixes)
        want = []
        first = 1
        while len(want) < quota:
            n = 1 << 18
            keys = np.frombuffer(oracle.chain_keys_mt(start, first, n), dtype=np.uint8).reshape(-1, 32)
            for i in range(n):
                k = bytes(keys[i])
                if fs.match(k) >= 0:
                    want.append((8 * (first + i), k))
                    if len(want) == quota:
                        break
            first += n
        assert want == out[sid], sid


def test_admission_by_memory(device):
    b = B.Batch(device, memory_budget=40_000, **SMALL)
    b.admit(1, workloads.seed(1), ["ab"], 1)  # a 16-bit index: 8 KiB
    with pytest.raises(N.OgError) as e:
        r = workloads.SplitMix64(3)
        b.admit(2, workloads.seed(2), [r.prefix(6, 6) for _ in range(3000)], 1)
    assert e.value.status == "OG_E_NOMEM"
    assert b.counts() == (1, 1)
    used, budget = b.memory()
    assert 0 < used <= budget == 40_000
    b.retire(1)
    assert b.memory()[0] == 0


def test_retire_mid_search_and_errors(device):
    b = B.Batch(device, **SMALL)
    b.admit(7, workloads.seed(7), ["abcdefg"], 1)
    b.admit(8, workloads.seed(8), ["ab"], 2)
    b.step()
    assert b.status(7).done == 0
    b.retire(7)
    with pytest.raises(N.OgError):
        b.status(7)
    with pytest.raises(N.OgError) as e:
        b.admit(8, workloads.seed(8), ["ab"], 2)
    assert e.value.status == "OG_E_STATE"
    with pytest.raises(N.OgError) as e:
        b.admit(9, workloads.seed(9), ["a0"], 2)
    assert e.value.status == "OG_E_FILTER"
    while b.running():
        b.step()
    assert len(b.results(8)) == 2


def test_tuner_records_a_shape_that_finds_the_same_hits(device, mixed, tmp_path, monkeypatch):
    """og_batch_tune walks inversion batch, slot pool and grid, records the
    fastest shape in tuning.yaml, and a batch created with zeros runs it; the
    hits of a search do not depend on the shape."""
    monkeypatch.setenv("ONION_GEN_TUNING_FILE", str(tmp_path / "tuning.yaml"))
    cfg, rate = B.tune(device, searches=16, max_step_ms=50.0)
    assert rate > 1e9
    assert cfg.half in (128, 256, 512) and cfg.slots % 128 == 0 and cfg.grid >= 1
    text = (tmp_path / "tuning.yaml").read_text()
    assert f"device/{device.name}/cuda-batch/0/" in text
    b = B.Batch(device)
    shape = b.shape()
    assert (shape.half, shape.slots, shape.grid, shape.rounds) == (cfg.half, cfg.slots, cfg.grid, cfg.rounds)
    b.close()
    out, _ = mixed
    tuned, _ = run_batch(device, SEARCHES, half=0, slots=0)
    assert tuned == out


SUFFIX_SEARCHES = [
    (201, workloads.suffix_filters(6, 8), 1),
    (202, workloads.suffix_filters(12, 8)[6:] + ["abc"], 2),
    (203, ["xy", "suffix:" + "q" * 6 + "id"], 3),
]


def test_suffix_searches_in_a_batch_agree_with_the_single_engine(device):
    """Suffix searches (alone and mixed with prefixes) in the batch find the
    same first hits as the single filter engine; every suffix hit's address
    really ends in its suffix."""
    b = B.Batch(device, half=256)
    for sid, filters, quota in SUFFIX_SEARCHES:
        b.admit(sid, workloads.seed(sid), filters, quota)
    steps = 0
    while b.running():
        b.step()
        steps += 1
        assert steps < 400
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import key

    for sid, filters, quota in SUFFIX_SEARCHES:
        got = b.results(sid)
        assert len(got) == quota
        cfg = N.EngineConfig(0, 256, 0, 1, 128, 0, 0)
        found, _, _ = run.device_search(device, workloads.seed(sid), filters, quota, config=cfg, max_advances=200)
        assert [(h.offset, h.packed) for h in found] == [key_of(h) for h in got], sid
        texts = F.FilterSet.parse_all(filters).texts()
        for h in got:
            t = texts[h.filter]
            addr = key.address(h.public_key)
            assert addr.endswith(t[7:]) if t.startswith("suffix:") else addr.startswith(t)
    b.close()


def test_a_leased_range_reports_every_block_s_finds_in_order(device):
    """run.search_lease: three blocks of a root seed searched at once; each
    find re-derives from its block's seed and matches a filter, and each
    block's finds are the single engine's first hits of that block's seed."""
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import key

    root = bytes(range(32))
    filters = ["ab", "q7"]
    finds = {}

    def report(block, offset):
        finds.setdefault(block, []).append(offset)
        return True

    steps = run.search_lease(device, root, 400, 3, filters, report, max_steps=6, half=64, slots=128 * 64)
    assert steps == 6 and sorted(finds) == [400, 401, 402]
    fs = F.FilterSet.parse_all(filters)
    cfg = N.EngineConfig(0, 64, 1024, 2, 128, 0, 0)
    for blk, offs in finds.items():
        assert offs == sorted(offs)
        seed = key.block_seed(root, blk)
        for off in offs[:20]:
            secret = key.expanded_secret_at_offset(seed, off)
            pk = key.pack(key.scalar_base_mult(secret[:32]))
            assert fs.match_address(pk) is not None
        found, _, _ = run.device_search(device, seed, filters, len(offs), config=cfg)
        assert [h.offset for h in found] == offs


def test_a_lease_split_over_ranks_finds_the_same_hits(device):
    """search_lease as rank 1 of 2 takes block 401 of the range 400..402 only;
    its finds are the same first hits of that block's seed that the whole
    range searched by one rank reports (both are prefixes of one sequence)."""
    root = bytes(range(32))
    filters = ["ab", "q7"]
    whole, part = {}, {}

    def into(d):
        return lambda block, offset: d.setdefault(block, []).append(offset) or True

    run.search_lease(device, root, 400, 3, filters, into(whole), max_steps=6, half=64, slots=128 * 64)
    run.search_lease(device, root, 400, 3, filters, into(part), max_steps=6, rank=1, world=2, half=64,
                     slots=128 * 64)
    assert sorted(part) == [401]
    n = min(len(part[401]), len(whole[401]))
    assert n > 0 and part[401][:n] == whole[401][:n]


def test_one_step_in_flight_agrees(device, mixed):
    """With one step queued at a time (no overlap of host and device work)
    the hits are the same as with two."""
    out, _ = mixed
    single, _ = run_batch(device, SEARCHES, inflight=1)
    assert single == out


def test_long_searches_at_a_larger_half_agree(device, mixed):
    """max_half lets a search whose expected work covers four steps of the
    whole pool run at a doubled inversion batch. Search 106 (one 5-symbol
    prefix, quota 1) expects 2^25 = 3.355e7 candidates: four steps of 8192
    slots at half 256 are 1.68e7, at half 512 3.358e7, so it runs at 256;
    search 103 (200 4-symbol prefixes, quota 8) expects 4.2e4 and stays at
    64. Their first hits do not change, nor do the others'."""
    out, _ = mixed
    b = B.Batch(device, **{**SMALL, "max_half": 512})
    for sid, prefixes, quota in SEARCHES:
        b.admit(sid, workloads.seed(sid), prefixes, quota)
    halves = {sid: b.status(sid).half for sid, _, _ in SEARCHES}
    assert halves[106] == 256 and halves[103] == 64, halves
    steps = 0
    while b.running():
        b.step()
        steps += 1
        assert steps < 5000
    got = {sid: [key_of(h) for h in b.results(sid)] for sid, _, _ in SEARCHES}
    for sid, _, quota in SEARCHES:
        st = b.status(sid)
        assert st.done == 1 and st.hits == quota and st.status == 0
        assert st.candidates == st.windows * (2 * halves[sid] + 1)
    b.close()
    assert got == out


def test_overflow_closes_the_batch(device):
    """More exact hits in a step than the room for them is an error, never
    a truncation; the batch then refuses further steps and admissions."""
    b = B.Batch(device, **{**SMALL, "max_hits": 4})
    b.admit(1, workloads.seed(1), ["ab", "cd"], 16)  # about 2000 hits a step
    with pytest.raises(N.OgError) as e:
        for _ in range(4):
            b.step()
    assert e.value.status == "OG_E_OVERFLOW"
    with pytest.raises(N.OgError) as e:
        b.step()
    assert e.value.status == "OG_E_STATE"
    with pytest.raises(N.OgError) as e:
        b.admit(2, workloads.seed(2), ["ab"], 1)
    assert e.value.status == "OG_E_STATE"
    b.close()


def test_a_hit_that_does_not_rederive_ends_only_its_search(device, mixed):
    """A re-derivation failure (planted on the host) ends that search with
    OG_E_VERIFY for the step it happens in; the other searches go on and
    find the same hits as in the mix without it, and later steps succeed."""
    out, _ = mixed
    b = B.Batch(device, **SMALL)
    for sid, prefixes, quota in SEARCHES:
        b.admit(sid, workloads.seed(sid), prefixes, quota)
    b.plant_mismatch(105)
    verify_errors = 0
    steps = 0
    while b.running():
        try:
            b.step()
        except N.OgError as e:
            assert e.status == "OG_E_VERIFY"
            verify_errors += 1
        steps += 1
        assert steps < 5000
    assert verify_errors == 1
    st = b.status(105)
    assert st.done == 1 and N.STATUS[st.status] == "OG_E_VERIFY" and st.hits < 16
    for sid, _, quota in SEARCHES:
        if sid == 105:
            continue
        assert b.status(sid).status == 0
        assert [key_of(h) for h in b.results(sid)] == out[sid], sid
    b.close()


def test_an_id_admitted_again_while_a_step_is_in_flight(device):
    """A search retired while it holds lanes in the step still in flight, and
    its id admitted again at once with other filters: the old search's hits
    in that step are not taken for the new one's, whose result equals a
    fresh run of it."""
    b = B.Batch(device, **SMALL)
    b.admit(5, workloads.seed(50), ["ab"], 50000)  # about 2000 hits a step, far from its quota
    b.admit(6, workloads.seed(6), ["q7"], 2)
    b.step()  # two steps launched, the first collected: search 5 has lanes in the second
    assert b.status(5).done == 0
    b.retire(5)
    b.admit(5, workloads.seed(5), ["cd"], 3)
    steps = 0
    while b.running():
        b.step()
        steps += 1
        assert steps < 5000
    assert b.status(5).status == 0 and b.status(6).status == 0
    got = [key_of(h) for h in b.results(5)]
    b.close()
    alone, _ = run_batch(device, [(5, ["cd"], 3)])
    assert got == alone[5]
