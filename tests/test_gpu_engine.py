"""Parity of the sm_100a engine with the CPU oracle (runs on a B200: -m gpu).

Every test drives the engine through the C ABI (libonion_gen_b200.so via
ctypes) and checks it against the oracle's restatement of the reference
engines on the same seeded inputs: bit-exact keys, exact offsets, exact
survivor sets.
"""
import json
import os

import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import gpu, key, workloads

pytestmark = pytest.mark.gpu


def cfg(scheme, half, lanes, rounds, dump=1, block=128, room=0, lanes_per_thread=0):
    return N.EngineConfig(scheme, half, lanes, rounds, block, dump, room, lanes_per_thread)


def oracle_start(oracle, seed):
    return oracle.scalar_base_mult(oracle.secret_scalar(seed))


def sorted_run(engine, advances=1):
    offs, keys = [], []
    for _ in range(advances):
        o, k = engine.advance_raw()
        offs.append(o)
        keys.append(k)
    o = np.concatenate(offs)
    k = np.concatenate(keys)
    order = np.argsort(o, kind="stable")
    return o[order], k[order]


def test_chain_config1_bit_exact_against_batch_engine(oracle, device):
    """4096 lanes x 256 steps, Z batch-inverted 256 at a time: all 2^20 keys
    equal src/batch.rs's BatchEngine(256) from the same base scalar."""
    start = oracle_start(oracle, workloads.seed(0))
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_CHAIN, 256, 4096, 1))
    assert eng.batch() == 1 << 20
    offs, keys = sorted_run(eng)
    assert np.array_equal(offs, 8 * np.arange(1 << 20, dtype=np.uint64))
    want = np.frombuffer(oracle.chain_keys(start, 256, 1 << 20), dtype=np.uint8).reshape(-1, 32)
    bad = np.nonzero((keys != want).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} keys differ, first at offset {8 * int(bad[0])}"
    # and 1024 of them against the reference's own verifier (tests/golden/config1_sample.json)
    sample = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config1_sample.json")))
    for i, pub in zip(sample["index"], sample["public"]):
        ref = bytearray(bytes.fromhex(pub))
        ref[31] &= 0x7F
        assert bytes(keys[i]) == bytes(ref), i


def test_paired_bit_exact_two_rounds(oracle, device):
    start = oracle_start(oracle, workloads.seed(0))
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, 128, 1024, 2))
    n = 1024 * 257 * 2
    assert eng.batch() == n
    offs, keys = sorted_run(eng)
    assert np.array_equal(offs, 8 * (1 + np.arange(n, dtype=np.uint64)))
    want = np.frombuffer(oracle.chain_keys_mt(start, 1, n), dtype=np.uint8).reshape(-1, 32)
    bad = np.nonzero((keys != want).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} keys differ, first at offset {int(offs[bad[0]])}"


@pytest.mark.parametrize("half,lanes,rounds", [(32, 256, 3), (1, 128, 2), (300, 384, 1), (1024, 256, 1), (2048, 128, 1)])
def test_paired_consecutive_advances_tile_the_range(oracle, device, half, lanes, rounds):
    """Two advances continue where the first stopped: no gap, no overlap."""
    start = oracle_start(oracle, workloads.seed(7))
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, half, lanes, rounds))
    offs, keys = sorted_run(eng, advances=2)
    n = 2 * lanes * (2 * half + 1) * rounds
    assert np.array_equal(offs, 8 * (1 + np.arange(n, dtype=np.uint64)))
    want = np.frombuffer(oracle.chain_keys_mt(start, 1, n), dtype=np.uint8).reshape(-1, 32)
    assert np.array_equal(keys, want)


@pytest.mark.parametrize("half,lanes,rounds", [(32, 256, 3), (1, 256, 2), (300, 768, 1), (2048, 256, 1)])
def test_two_lanes_per_thread_tile_the_range(oracle, device, half, lanes, rounds):
    """The two-lanes-per-thread kernel (one inversion shared by a thread's
    lanes) covers the same candidates bit for bit, advance after advance."""
    start = oracle_start(oracle, workloads.seed(8))
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, half, lanes, rounds, lanes_per_thread=2))
    assert eng.shape().lanes_per_thread == 2
    offs, keys = sorted_run(eng, advances=2)
    n = 2 * lanes * (2 * half + 1) * rounds
    assert np.array_equal(offs, 8 * (1 + np.arange(n, dtype=np.uint64)))
    want = np.frombuffer(oracle.chain_keys_mt(start, 1, n), dtype=np.uint8).reshape(-1, 32)
    assert np.array_equal(keys, want)


def test_two_lanes_per_thread_filtered_equals_one(device):
    """With a bitmap, the two kernels return the same survivors."""
    fs = F.FilterSet.parse_all(["ab", "q7", "zz2"])
    words, bits = fs.index_words()
    start = key.start_point(workloads.seed(9))
    got = []
    for lpt in (1, 2):
        eng = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits,
                         config=cfg(N.SCHEME_PAIRED, 256, 8192, 1, dump=0, lanes_per_thread=lpt))
        offs, keys = sorted_run(eng, advances=2)
        eng.close()
        got.append((offs.tolist(), keys.tobytes()))
    assert got[0] == got[1] and len(got[0][0]) > 1000


def test_lanes_per_thread_is_checked(device):
    start = key.start_point(workloads.seed(9))
    with pytest.raises(N.OgError) as e:
        gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, 64, 256, 1, lanes_per_thread=3))
    assert e.value.status == "OG_E_ARG"
    with pytest.raises(N.OgError) as e:
        gpu.Engine(device, start, config=cfg(N.SCHEME_CHAIN, 64, 256, 1, lanes_per_thread=2))
    assert e.value.status == "OG_E_ARG"


def test_chain_two_advances_continue(oracle, device):
    start = oracle_start(oracle, workloads.seed(3))
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_CHAIN, 64, 256, 2))
    offs, keys = sorted_run(eng, advances=2)
    n = 2 * 256 * 64 * 2
    assert np.array_equal(offs, 8 * np.arange(n, dtype=np.uint64))
    want = np.frombuffer(oracle.chain_keys_mt(start, 0, n), dtype=np.uint8).reshape(-1, 32)
    assert np.array_equal(keys, want)


def test_reference_pair_engine_keys_appear_at_their_deltas(oracle, device):
    """The reference's own paired CPU engine (src/pairs.rs) and this engine
    agree on the key of every delta both produce."""
    start = oracle_start(oracle, workloads.seed(11))
    ref_keys, deltas = oracle.pair_keys(start, 96, 4)
    ref = np.frombuffer(ref_keys, dtype=np.uint8).reshape(-1, 32)
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, 96, 128, 1))
    offs, keys = sorted_run(eng)
    index = {int(o): i for i, o in enumerate(offs)}
    for d, k in zip(deltas, ref):
        assert np.array_equal(keys[index[int(d)]], k), f"delta {int(d)}"


def filtered_parity(oracle, device, prefixes, bits, half, lanes, rounds, seed_i):
    start = oracle_start(oracle, workloads.seed(seed_i))
    fs = F.FilterSet.parse_all(prefixes, bits=bits)
    words, b = fs.index_words()
    ofs = oracle.FilterSet(prefixes, bits=bits)
    assert b == ofs.bits and np.array_equal(words, ofs.words())
    eng = gpu.Engine(device, start, bitmap=words, bitmap_bits=b, config=cfg(N.SCHEME_PAIRED, half, lanes, rounds, dump=0))
    offs, keys = sorted_run(eng)
    n = eng.batch()
    # the oracle's survivors over the same range, in chunks
    want = []
    chunk = 1 << 22
    for lo in range(0, n, chunk):
        cnt = min(chunk, n - lo)
        ks = np.frombuffer(oracle.chain_keys_mt(start, 1 + lo, cnt), dtype=np.uint8).reshape(-1, 32)
        head = ks[:, :4].astype(np.uint32)
        h32 = (head[:, 0] << 24) | (head[:, 1] << 16) | (head[:, 2] << 8) | head[:, 3]
        slot = (h32 >> (32 - b)).astype(np.uint64)
        hit = ((words[slot >> 6] >> (slot & 63)) & 1).astype(bool)
        for i in np.nonzero(hit)[0]:
            want.append((8 * (1 + lo + int(i)), bytes(ks[i])))
    got = [(int(o), bytes(k)) for o, k in zip(offs, keys)]
    assert got == want
    return start, fs, got


def test_paired_bitmap_survivors_equal_oracle(oracle, device):
    """A 3-symbol prefix on a 16-bit index over 2^24 candidates: the exact
    set of bitmap survivors, offsets and keys."""
    start, fs, got = filtered_parity(oracle, device, ["abc"], 0, 128, 2048, 32, 1)
    assert 300 < len(got) < 800  # 2^24 / 2^15 = 512 expected
    seed = workloads.seed(1)
    for off, packed in got:
        pk, _ = key.check_hit(seed, off, packed)
        assert pk[:31] == packed[:31]


def test_paired_wide_bitmap_many_prefixes(oracle, device):
    """Config 3 on its parity sub-range: 10,000 prefixes of 3..8 symbols, a
    24-bit index at ~5% occupancy, the first 16.8 M candidates (2^24 and a
    little more): the same ~840 k survivors as the oracle's, and the same
    exact matches."""
    prefixes = workloads.config3_prefixes()
    start, fs, got = filtered_parity(oracle, device, prefixes, 0, 128, 4096, 16, 0)
    assert fs.bits == 24 and len(got) > 700_000
    packed = np.frombuffer(b"".join(p for _, p in got), dtype=np.uint8).reshape(-1, 32)
    ofs = oracle.FilterSet(prefixes)
    m = fs.match_many(packed)
    for k in range(0, len(got), 97):
        assert m[k] == ofs.match(got[k][1])
    for off, p in got[:200]:
        key.check_hit(workloads.seed(0), off, p)


def test_overflow_is_an_error_not_a_truncation(oracle, device):
    start = oracle_start(oracle, workloads.seed(0))
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, 32, 128, 1, room=100))
    with pytest.raises(N.OgError) as e:
        eng.advance()
    assert e.value.status == "OG_E_OVERFLOW"
    with pytest.raises(N.OgError) as e:
        eng.advance()
    assert e.value.status == "OG_E_STATE"


def test_reference_shaped_constructor_and_tuning_cache(oracle, device, tmp_path, monkeypatch):
    """og_engine_new with threads=0 walks shapes, records the fastest in
    tuning.yaml (format 1, the reference's key), and reuses it."""
    path = tmp_path / "tuning.yaml"
    monkeypatch.setenv("ONION_GEN_TUNING_FILE", str(path))
    start = oracle_start(oracle, workloads.seed(0))
    fs = F.FilterSet.parse_all([workloads.config2_prefix()])
    words, bits = fs.index_words()
    eng = gpu.Engine(device, start, threads=0, bitmap=words, bitmap_bits=bits)
    text = path.read_text()
    assert text.startswith("format: 1\nentries:\n")
    assert f"device/{device.name}/cuda/0/" in text
    shape = eng.shape()
    eng2 = gpu.Engine(device, start, threads=0, bitmap=words, bitmap_bits=bits)
    assert (eng2.shape().half, eng2.shape().lanes) == (shape.half, shape.lanes)
    # survivors of the tuned engine are real keys
    for s in eng2.advance()[:50]:
        key.check_hit(workloads.seed(0), s.offset, s.packed)


def test_threads_argument_is_lanes(oracle, device):
    start = oracle_start(oracle, workloads.seed(0))
    fs = F.FilterSet.parse_all(["ab"])
    words, bits = fs.index_words()
    eng = gpu.Engine(device, start, threads=1000, bitmap=words, bitmap_bits=bits)
    assert eng.threads() == 1024  # rounded up to whole blocks
    survivors = eng.advance()
    assert survivors
    for s in survivors[:100]:
        key.check_hit(workloads.seed(0), s.offset, s.packed)
        assert fs.match_key(s.packed) is not None


def test_paired_pattern_bitmap_survivors_equal_oracle(oracle, device):
    """Prefixes with wildcards and classes fill the same bitmap as the
    oracle's pattern_slots, and the same candidates survive."""
    start, fs, got = filtered_parity(oracle, device, ["a?c", "[xyz]2", "k[a-e]?m", "q7", "mm[2-7]"], 16, 128, 2048,
                                     8, 2)
    assert len(got) > 100


@pytest.mark.parametrize("bits", [8, 26, 32])
def test_bitmap_width_extremes(oracle, device, bits):
    """The narrowest index the engine takes, a 64 MiB one and the widest
    (32 bits, 512 MiB; the reference's --index-bits range is 8..32): the
    same survivors as the oracle's."""
    prefixes = ["abc", "q7x"]
    start, fs, got = filtered_parity(oracle, device, prefixes, bits, 64, 1024, 4, 4)
    assert fs.bits == bits and len(got) > 0


def test_default_shape_is_eight_blocks_per_resident_cta(oracle, device):
    """og_engine_resident_lanes reports one wave of the paired kernel; an
    engine built with lanes 0 takes eight blocks of 128 per resident CTA and
    half 2048, and its first advance tiles the range."""
    resident = gpu.resident_lanes(device)
    assert resident % (128 * device.sms) == 0 and resident >= 128 * device.sms
    start = oracle_start(oracle, workloads.seed(2))
    fs = F.FilterSet.parse_all(["abcdefg"])
    words, bits = fs.index_words()
    eng = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg(N.SCHEME_PAIRED, 0, 0, 1, dump=0))
    shape = eng.shape()
    assert shape.half == 2048 and eng.threads() == 8 * resident
    assert eng.batch() == 8 * resident * (2 * 2048 + 1)
    for s in eng.advance()[:20]:
        key.check_hit(workloads.seed(2), s.offset, s.packed)
    with pytest.raises(N.OgError):
        gpu.resident_lanes(device, scheme=7)


def test_reference_gpu_harness_case(device):
    """The reference's own device check (benches/gpu-chain.rs:15-94): filter
    "abc", seed [7; 32], 2^14 threads, four launches through the
    reference-shaped constructor. Every survivor is re-derived from its
    offset alone and must equal the device's key (sign bit masked); the
    index must let something through; an exact match spells "abc"."""
    seed = bytes([7] * 32)
    fs = F.FilterSet.parse_all(["abc"])
    words, bits = fs.index_words()
    eng = gpu.Engine(device, key.start_point(seed), threads=1 << 14, bitmap=words, bitmap_bits=bits)
    assert eng.threads() == 1 << 14
    examined, offsets, confirmed = 0, set(), 0
    for _ in range(4):
        hits = eng.advance()
        examined += eng.batch()
        for h in hits:
            pk, _ = key.check_hit(seed, h.offset, h.packed)
            assert pk[:31] == h.packed[:31] and (pk[31] & 0x7F) == h.packed[31]
            assert h.offset % 8 == 0 and 0 < h.offset <= 8 * examined and h.offset not in offsets
            offsets.add(h.offset)
            if fs.match_key(h.packed) is not None:
                confirmed += 1
                assert key.address(pk).startswith("abc")
    assert examined == 4 * eng.batch() and len(offsets) > 0
    # a 15-bit literal on its index: about examined / 2^15 exact matches
    assert 0.5 * examined / 2**15 < confirmed < 1.5 * examined / 2**15


def test_default_shape_for_a_dense_index(device):
    """A set that lets 5 % of candidates through (config 3): the default keeps
    eight waves of lanes and shortens the inversion batch until one advance's
    expected survivors fit 2^26 records; the room holds the expected count
    plus eight standard deviations; an advance returns about that many."""
    resident = gpu.resident_lanes(device)
    fs = F.FilterSet.parse_all(workloads.config3_prefixes())
    words, bits = fs.index_words()
    occ = fs.occupancy()
    half = 2048
    while half > 256 and 8 * resident * (2 * half + 1) * occ > 2**26:
        half //= 2
    eng = gpu.Engine(device, key.start_point(workloads.seed(0)), bitmap=words, bitmap_bits=bits,
                     config=cfg(N.SCHEME_PAIRED, 0, 0, 1, dump=0))
    assert eng.shape().half == half < 2048 and eng.threads() == 8 * resident
    mu = eng.batch() * occ
    assert mu + 7.9 * mu**0.5 < eng.room() < mu + 8.1 * mu**0.5 + 1100
    o, k = eng.advance_raw()
    assert abs(len(o) - mu) < 6 * mu**0.5
    for i in range(0, len(o), len(o) // 50):
        key.check_hit(workloads.seed(0), int(o[i]), bytes(k[i]))


@pytest.mark.parametrize("block", [32, 96])
def test_paired_smaller_blocks_tile_the_range(oracle, device, block):
    """Blocks of 32 and 96 threads (the ABI takes any multiple of 32 up to
    128): the persistent CTAs, the parked centres and the scratch slots are
    per block, and two advances still tile the range bit-exactly."""
    start = oracle_start(oracle, workloads.seed(13))
    lanes = 4 * 96
    eng = gpu.Engine(device, start, config=cfg(N.SCHEME_PAIRED, 48, lanes, 2, block=block))
    assert eng.shape().block == block and eng.threads() == lanes
    offs, keys = sorted_run(eng, advances=2)
    n = 2 * lanes * (2 * 48 + 1) * 2
    assert np.array_equal(offs, 8 * (1 + np.arange(n, dtype=np.uint64)))
    want = np.frombuffer(oracle.chain_keys_mt(start, 1, n), dtype=np.uint8).reshape(-1, 32)
    assert np.array_equal(keys, want)
