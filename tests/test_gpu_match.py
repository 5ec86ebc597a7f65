"""Device-side exact match of the single engine (og_engine_match_on_device,
og_engine_advance_matches) against the host's FilterSet::match_key over the
same engine's survivors (runs on a B200: -m gpu).

Two engines of one shape from one start: the first returns its bitmap
survivors and the host matches them (run::device_worker, src/run.rs:1081-1085);
the second matches on the device. The two match lists must be equal —
offsets, keys and filter indices — including filters longer than the 12
symbols the device tables hold, which the host confirms.
"""
import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import gpu, key, workloads

pytestmark = pytest.mark.gpu

HALF, LANES, ROUNDS = 128, 1024, 8
SLOTS = 2 * HALF + 1


def cfg(dump=0):
    return N.EngineConfig(N.SCHEME_PAIRED, HALF, LANES, ROUNDS, 128, dump, 0)


def key_at(seed, offset):
    secret = key.expanded_secret_at_offset(seed, offset)
    return key.pack(key.scalar_base_mult(secret[:32]))


def host_matches(eng, fs, advances):
    out = []
    for _ in range(advances):
        o, k = eng.advance_raw()
        m = fs.match_many(k)
        for j in np.nonzero(m >= 0)[0]:
            out.append((int(o[j]), bytes(k[j]), int(m[j])))
    return sorted(out)


def device_matches(eng, advances):
    out = []
    for _ in range(advances):
        o, k, f = eng.advance_matches_raw()
        out.extend((int(a), bytes(b), int(c)) for a, b, c in zip(o, k, f))
    return sorted(out)


def test_device_match_equals_host_match(device):
    seed = workloads.seed(0)
    start = key.start_point(seed)
    # config 3's prefixes plus long filters built from a key the first
    # advance examines: one that matches it on 14 symbols, one that shares
    # its first 12 symbols and differs after (the device cannot tell them
    # apart), and one of 20 symbols that matches
    off = 8 * (5 * SLOTS + 1 + 17)
    text = key.address(key_at(seed, off))
    decoy = text[:12] + ("a" if text[12] != "a" else "b") + text[13]
    prefixes = workloads.config3_prefixes(2000) + [text[:14], decoy, text[:20]]
    fs = F.FilterSet.parse_all(prefixes)
    words, bits = fs.index_words()
    plain = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    want = host_matches(plain, fs, 2)
    plain.close()
    matched = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    matched.match_on_device(fs)
    got = device_matches(matched, 2)
    matched.close()
    assert len(want) > 1000
    assert got == want
    # the constructed key is found, owned by its 14-symbol filter (the
    # 20-symbol one is absorbed by it)
    texts = fs.texts()
    hit = [g for g in got if g[0] == off]
    assert len(hit) == 1 and texts[hit[0][2]] == text[:14]
    assert decoy in texts
    for o, packed, f in got[:100]:
        pk, _ = key.check_hit(seed, o, packed)
        assert key.address(pk).startswith(texts[f])


def test_device_match_refuses_a_different_filter_set(device):
    start = key.start_point(workloads.seed(0))
    fs = F.FilterSet.parse_all(["abc"])
    other = F.FilterSet.parse_all(["abd"])
    words, bits = fs.index_words()
    eng = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    with pytest.raises(N.OgError) as e:
        eng.advance_matches_raw()
    assert e.value.status == "OG_E_STATE"
    with pytest.raises(N.OgError) as e:
        eng.match_on_device(other)
    assert e.value.status == "OG_E_ARG"
    eng.match_on_device(fs)
    o, k, f = eng.advance_matches_raw()
    assert all(fs.match_key(bytes(p)) == 0 for p in k)
    dump = gpu.Engine(device, start, config=cfg(dump=1))
    with pytest.raises(N.OgError) as e:
        dump.match_on_device(fs)
    assert e.value.status == "OG_E_STATE"


def test_run_driver_finds_the_same_hits_with_the_device_match(device):
    from onion_gen_b200 import run

    searches = [s for s in workloads.config4_searches() if s.quota / sum(32.0 ** -len(p) for p in s.prefixes) < 2e7]
    assert len(searches) >= 2
    for s in searches[:3]:
        host, ex_h, adv_h = run.device_search(device, s.seed, s.prefixes, s.quota, config=cfg(), max_advances=40)
        dev, ex_d, adv_d = run.device_search(device, s.seed, s.prefixes, s.quota, config=cfg(), max_advances=40,
                                             device_match=True)
        assert len(host) == s.quota
        assert dev == host and (ex_d, adv_d) == (ex_h, adv_h)


def test_device_match_of_patterns_equals_host_match(device):
    """Wildcards and classes, walked on the device after the literal buckets,
    in the same order the host's match_key walks them."""
    start = key.start_point(workloads.seed(5))
    fs = F.FilterSet.parse_all(["a?c", "[xyz]2", "k[a-e]?m", "q7", "mm[2-7]", "a", "[b-d]??x"])
    words, bits = fs.index_words()
    plain = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    want = host_matches(plain, fs, 2)
    plain.close()
    matched = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    matched.match_on_device(fs)
    got = device_matches(matched, 2)
    matched.close()
    texts = fs.texts()
    assert got == want
    assert {texts[f] for _, _, f in got} >= {"a", "q7"} and any("?" in texts[f] or "[" in texts[f] for _, _, f in got)


def test_launch_and_collect_pipeline_equals_advance(device):
    """Two advances in flight (og_engine_launch / og_engine_collect) give the
    same survivors, in launch order, as advance after advance; so do the
    matching halves; misuse is an error, not a hang."""
    start = key.start_point(workloads.seed(6))
    fs = F.FilterSet.parse_all(["ab", "x7", "suffix:" + "b" * 7 + "qd"])
    a = gpu.Engine(device, start, filters=fs, config=cfg())
    want = [a.advance_raw() for _ in range(4)]
    a.close()
    b = gpu.Engine(device, start, filters=fs, config=cfg())
    with pytest.raises(N.OgError) as e:
        b.collect_raw()
    assert e.value.status == "OG_E_STATE"
    got = []
    b.launch()
    b.launch()
    with pytest.raises(N.OgError) as e:
        b.launch()
    assert e.value.status == "OG_E_STATE"
    with pytest.raises(N.OgError) as e:
        b.advance_raw()
    assert e.value.status == "OG_E_STATE"
    got.append(b.collect_raw())
    b.launch()
    got.append(b.collect_raw())
    got.append(b.collect_raw())
    b.launch()
    got.append(b.collect_raw())
    # survivors are appended by atomics, so each advance's set is compared in offset order
    for (wo, wk), (go, gk) in zip(want, got):
        i, j = np.argsort(wo), np.argsort(go)
        assert np.array_equal(wo[i], go[j]) and np.array_equal(wk[i], gk[j])
    b.close()
    # the matching halves
    c = gpu.Engine(device, start, filters=fs, config=cfg())
    want = [c.advance_matches_raw() for _ in range(3)]
    c.close()
    d = gpu.Engine(device, start, filters=fs, config=cfg())
    d.launch_matches()
    d.launch_matches()
    got = [d.collect_matches_raw()]
    d.launch_matches()
    got += [d.collect_matches_raw(), d.collect_matches_raw()]
    for w, g in zip(want, got):
        i, j = np.argsort(w[0]), np.argsort(g[0])
        assert all(np.array_equal(x[i], y[j]) for x, y in zip(w, g))
    assert sum(len(w[0]) for w in want) > 0
    d.close()


@pytest.mark.parametrize("device_match", [False, True])
def test_full_address_filters(device, device_match):
    """Filters past the key-only symbols: a whole 56-symbol address and a
    53-symbol prefix (sign bit and checksum symbols included), each built
    from a key the first advance examines, and a whole address one symbol
    off. The run driver finds exactly the two keys, confirmed on their
    addresses, with the host match and with the device match."""
    from onion_gen_b200 import run

    seed = workloads.seed(9)
    off1, off2 = 8 * (3 * SLOTS + 1 + 40), 8 * (700 * SLOTS + 1 + 200)
    a1, a2 = key.address(key_at(seed, off1)), key.address(key_at(seed, off2))
    decoy = a1[:30] + ("a" if a1[30] != "a" else "b") + a1[31:]
    filters = [a1, a2[:53], decoy]
    found, examined, advances = run.device_search(device, seed, filters, 3, config=cfg(), max_advances=1,
                                                  device_match=device_match)
    assert advances == 1 and examined == LANES * ROUNDS * SLOTS
    texts = F.FilterSet.parse_all(filters).texts()
    assert [(h.offset, texts[h.filter]) for h in found] == [(off1, a1), (off2, a2[:53])]
    assert key.address(found[0].public_key) == a1


def test_chain_scheme_device_match_equals_host_match(device):
    """The chain scheme (scheme 1) with the device match: the same matches,
    offsets and filter indices as the host's match of its survivors, on
    literal prefixes of config 3 plus patterns."""
    start = key.start_point(workloads.seed(4))
    fs = F.FilterSet.parse_all(workloads.config3_prefixes(1500) + ["a?c", "[xyz]2k"])
    words, bits = fs.index_words()
    chain = N.EngineConfig(N.SCHEME_CHAIN, 256, 1024, 2, 128, 0, 0)
    plain = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=chain)
    want = host_matches(plain, fs, 2)
    plain.close()
    matched = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=chain)
    matched.match_on_device(fs)
    got = device_matches(matched, 2)
    matched.close()
    assert len(want) > 100 and got == want
    for o, packed, f in got[:50]:
        pk, _ = key.check_hit(workloads.seed(4), o, packed)
        assert fs.match_address(pk) == f


def view_matches(eng, advances):
    out = []
    for _ in range(advances):
        eng.launch_matches()
        o, k, f = eng.collect_matches_view_raw()
        out.extend((int(a), bytes(b), int(c)) for a, b, c in zip(o, k, f))
    return sorted(out)


def test_matches_view_equals_host_match(device):
    """og_engine_collect_matches_view leaves each advance's matches in the
    engine's pinned memory in og_match's layout, their offsets decoded on the
    device: they equal the host's match of the same engine's survivors,
    filters longer than the device tables confirmed on the host included
    (the decoy that shares 12 symbols is dropped). With two advances in
    flight the views come back in launch order."""
    seed = workloads.seed(0)
    start = key.start_point(seed)
    off = 8 * (5 * SLOTS + 1 + 17)
    text = key.address(key_at(seed, off))
    decoy = text[:12] + ("a" if text[12] != "a" else "b") + text[13]
    fs = F.FilterSet.parse_all(workloads.config3_prefixes(2000) + [text[:14], decoy])
    words, bits = fs.index_words()
    plain = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    want = host_matches(plain, fs, 3)
    plain.close()
    v = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    v.match_on_device(fs)
    got = view_matches(v, 3)
    v.close()
    assert len(want) > 1000 and got == want
    assert [g for g in got if g[0] == off][0][2] == fs.texts().index(text[:14])
    # two in flight: launch, launch, view, launch, view, view
    w = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    w.match_on_device(fs)
    w.launch_matches()
    w.launch_matches()
    views = [w.collect_matches_view_raw()]
    w.launch_matches()
    views += [w.collect_matches_view_raw(), w.collect_matches_view_raw()]
    w.close()
    flat = sorted((int(a), bytes(b), int(c)) for o, k, f in views for a, b, c in zip(o, k, f))
    assert flat == want
    # each advance's matches lie in its own range of offsets, in launch order
    tops = [int(o.max()) for o, _, _ in views]
    bottoms = [int(o.min()) for o, _, _ in views]
    assert tops[0] < bottoms[1] and tops[1] < bottoms[2]
    with pytest.raises(N.OgError) as e:
        w2 = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
        try:
            w2.match_on_device(fs)
            w2.launch()
            w2.collect_matches_view()
        finally:
            w2.close()
    assert e.value.status == "OG_E_STATE"
