"""Suffix filters on the device (runs on a B200: -m gpu).

The engine built from a filter set (og_engine_new_filters) lets a candidate
through its suffix bitmap exactly when the oracle's restatement of the
reference's suffix index does, and its device match (the key recomputed from
the offset, sign bit and SHA3-256 checksum included) returns exactly the
survivors whose full address the host finds matching: offsets, keys and
filter indices.
"""
import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import gpu, key, workloads

pytestmark = pytest.mark.gpu

ALPHABET = "abcdefghijklmnopqrstuvwxyz234567"


def cfg(scheme=N.SCHEME_PAIRED, half=128, lanes=1024, rounds=16):
    return N.EngineConfig(scheme, half, lanes, rounds, 128, 0, 0)


def full_key(seed, offset):
    secret = key.expanded_secret_at_offset(seed, offset)
    return key.pack(key.scalar_base_mult(secret[:32]))


def suffix_slots(keys, bits):
    tail = keys[:, 24:32].astype(np.uint64)
    w = np.zeros(len(keys), dtype=np.uint64)
    for j in range(8):
        w = (w << np.uint64(8)) | tail[:, j]
    return (w >> np.uint64(1)) & np.uint64((1 << bits) - 1)


def eight_symbol_suffixes(n=40):
    return ["suffix:" + "".join(ALPHABET[(i * 5 + j * 7) % 32] for j in range(6)) + "ad" for i in range(n)]


def test_suffix_survivors_equal_the_oracle(oracle, device):
    seed = workloads.seed(2)
    start = key.start_point(seed)
    fs = F.FilterSet.parse_all(eight_symbol_suffixes())
    words, bits = fs.suffix_index_words()
    o = oracle.SuffixSet([t[7:] for t in fs.texts()])
    assert bits == o.bits and np.array_equal(words, o.words())
    eng = gpu.Engine(device, start, filters=fs, config=cfg())
    offs, keys = eng.advance_raw()
    n = eng.batch()
    order = np.argsort(offs, kind="stable")
    got = [(int(offs[i]), bytes(keys[i])) for i in order]
    ks = np.frombuffer(oracle.chain_keys_mt(start, 1, n), dtype=np.uint8).reshape(-1, 32)
    slot = suffix_slots(ks, bits)
    hit = ((words[slot >> np.uint64(6)] >> (slot & np.uint64(63))) & np.uint64(1)).astype(bool)
    want = [(8 * (1 + int(i)), bytes(ks[i])) for i in np.nonzero(hit)[0]]
    assert len(want) > 1000
    assert got == want


def host_matches(seed, fs, offs, keys):
    out = []
    for o, k in zip(offs, keys):
        pk, _ = key.check_hit(seed, int(o), bytes(k))
        m = fs.match_address(pk)
        if m is not None:
            out.append((int(o), bytes(k), m))
    return sorted(out)


@pytest.mark.parametrize("scheme,half,rounds", [(N.SCHEME_PAIRED, 128, 16), (N.SCHEME_CHAIN, 256, 4)])
def test_device_suffix_match_equals_the_host(device, scheme, half, rounds):
    seed = workloads.seed(3)
    start = key.start_point(seed)
    shape = cfg(scheme, half, 1024, rounds)
    # a target the first advance examines, matched through its sign bit
    # (symbol 49) and checksum (symbols 51..55), and a decoy that differs
    # from it only in the sign bit's place: same bitmap slot, no match
    probe = gpu.Engine(device, start, config=N.EngineConfig(scheme, half, 1024, rounds, 128, 1, 0))
    n = probe.batch()
    probe.close()
    off = 8 * (n // 3 + (1 if scheme == N.SCHEME_PAIRED else 0))
    addr = key.address(full_key(seed, off))
    target = "suffix:" + addr[46:]
    decoy = "suffix:" + addr[46:49] + ALPHABET[ALPHABET.index(addr[49]) ^ 2] + addr[50:]
    filters = eight_symbol_suffixes(24) + [target, decoy, "ab", "zq7"]
    fs = F.FilterSet.parse_all(filters)
    texts = fs.texts()
    a = gpu.Engine(device, start, filters=fs, config=shape)
    offs, keys = a.advance_raw()
    a.close()
    want = host_matches(seed, fs, offs, keys)
    b = gpu.Engine(device, start, filters=fs, config=shape)
    o, k, f = b.advance_matches_raw()
    b.close()
    got = sorted((int(x), bytes(y), int(z)) for x, y, z in zip(o, k, f))
    assert got == want
    assert any(g[2] < fs.prefix_count() for g in got), "no prefix match to compare"
    hit = [g for g in got if g[0] == off]
    assert len(hit) == 1 and texts[hit[0][2]] == target
    assert texts.index(decoy) not in [g[2] for g in got if g[0] == off]


def test_an_engine_without_suffix_bitmap_refuses_a_suffix_set(device):
    start = key.start_point(workloads.seed(0))
    fs = F.FilterSet.parse_all(["abc"])
    sfx = F.FilterSet.parse_all(["abc"] + eight_symbol_suffixes(2))
    words, bits = fs.index_words()
    eng = gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg())
    with pytest.raises(N.OgError) as e:
        eng.match_on_device(sfx)
    assert e.value.status == "OG_E_ARG"


def test_run_driver_with_a_prefix_and_a_suffix(device):
    """The package's front door on a mixed set, as a user calls it."""
    from onion_gen_b200 import run

    hits, examined, advances = run.device_search(device, workloads.seed(0), ["abcd", "suffix:zzzzzzzqd"], quota=2)
    assert len(hits) == 2 and advances >= 1 and examined > 0
    for h in hits:
        addr = key.address(h.public_key)
        assert addr.startswith("abcd") or addr.endswith("zzzzzzzqd")
