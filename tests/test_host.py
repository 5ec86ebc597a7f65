"""The engine's host code through the C ABI, no GPU: keys, re-derivation,
addresses, filters and the bitmap, against the golden fixtures and the oracle."""
import json
import math
import os
import random

import numpy as np
import pytest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
B = bytes.fromhex


def test_keys_against_golden(native):
    key = native.key
    for k in GOLDEN["keys"]:
        seed = B(k["seed"])
        assert key.secret_scalar(seed).hex() == k["scalar"]
        assert key.public_key(seed).hex() == k["public"]
        assert key.hostname(B(k["public"])) == k["address"]


def test_offsets_against_golden(native):
    key = native.key
    for o in GOLDEN["offsets"]:
        pk, sec = key.check_hit(B(o["seed"]), o["offset"], B(o["packed"]))
        assert pk.hex() == o["public"]
        assert sec[:32] == key.expanded_secret_at_offset(B(o["seed"]), o["offset"])[:32]


def test_check_hit_rejects_a_wrong_key(native):
    """A corrupted survivor (offset or key) is refused, never accepted:
    faults made on the host (src/run.rs:1101-1104 counts these)."""
    key = native.key
    o = GOLDEN["offsets"][3]
    seed, off, packed = B(o["seed"]), o["offset"], bytearray(B(o["packed"]))
    key.check_hit(seed, off, bytes(packed))
    with pytest.raises(native._native.OgError) as e:
        key.check_hit(seed, off + 8, bytes(packed))
    assert e.value.status == "OG_E_VERIFY"
    packed[5] ^= 1
    with pytest.raises(native._native.OgError):
        key.check_hit(seed, off, bytes(packed))
    # the sign bit is not compared (the device leaves it clear)
    p2 = bytearray(B(o["packed"]))
    p2[31] |= 0x80
    key.check_hit(seed, off, bytes(p2))


def test_host_agrees_with_oracle_on_random_seeds(native, oracle):
    key = native.key
    rng = random.Random(5)
    for _ in range(100):
        seed = bytes(rng.getrandbits(8) for _ in range(32))
        assert key.public_key(seed) == oracle.public_key(seed)
        off = 8 * rng.getrandbits(40)
        assert key.expanded_secret_at_offset(seed, off) == oracle.expanded_secret_at_offset(seed, off)
        root = bytes(rng.getrandbits(8) for _ in range(32))
        assert key.block_seed(root, off) == oracle.block_seed(root, off)


def test_scalar_base_mult_agrees(native, oracle):
    rng = random.Random(9)
    for _ in range(50):
        s = bytes(rng.getrandbits(8) for _ in range(32))
        assert native.key.pack(native.key.scalar_base_mult(s)) == oracle.pack(oracle.scalar_base_mult(s))


FILTER_SETS = [
    ["abc"],
    ["abcd", "abcdef", "zzzz", "qrst", "mnopqr", "a" * 20],
    ["ABC", "  prefix:xyz2 ", "^^q7", "abd", "abc"],
    ["a" * 49, "b" * 56, "c"],
]


@pytest.mark.parametrize("filters", FILTER_SETS)
@pytest.mark.parametrize("bits", [0, 12, 16, 20, 24])
def test_filter_sets_agree_with_oracle(native, oracle, filters, bits):
    try:
        mine = native.filter.FilterSet.parse_all(filters, bits=bits)
    except native._native.OgError:
        with pytest.raises(ValueError):
            oracle.FilterSet(filters, bits=bits)
        return
    ref = oracle.FilterSet(filters, bits=bits)
    assert mine.texts() == ref.canonical()
    w, b = mine.index_words()
    assert b == ref.bits
    assert np.array_equal(w, ref.words())
    assert abs(mine.occupancy() - ref.occupancy()) < 1e-12
    rng = random.Random(bits)
    for i in range(3000):
        packed = bytes(rng.getrandbits(8) for _ in range(32))
        if i % 2 == 0:
            # force a match on one filter's leading bytes
            t = ref.canonical()[(i // 2) % len(ref)]
            raw, _ = oracle.base32_decode_bits(t[:49])
            n = (5 * min(len(t), 49) + 7) // 8
            packed = raw[:n] + packed[n:]
        a = mine.match_key(packed)
        r = ref.match(packed)
        assert (a is None and r < 0) or a == r


def test_filter_errors(native):
    F = native.filter.FilterSet
    E = native._native.OgError
    for bad in ["", "^", "ab0c", "a" * 57, "suffix:abd", "contains:abc", "regex:^ab", "a[bc", "??"]:
        with pytest.raises(E) as e:
            F.parse_all([bad])
        assert e.value.status == "OG_E_FILTER"


def test_saturated_index_is_discarded(native):
    # src/filter.rs a_saturated_index_is_discarded
    alphabet = "abcdefghijklmnopqrstuvwxyz234567"
    F = native.filter.FilterSet
    assert F.parse_all(["ab"]).bits == 16
    pairs = [a + b for a in alphabet for b in alphabet]
    with pytest.raises(native._native.OgError):
        F.parse_all(pairs)
    three = [alphabet[i % 32] + alphabet[(i // 32) % 32] + alphabet[(i // 1024 + 7) % 32] for i in range(1000)]
    assert F.parse_all(three).bits >= 16


def test_index_width_and_size(native):
    # src/filter.rs index_size_follows_its_width; narrowest_acceptable picks 16 for few filters
    F = native.filter.FilterSet
    w, b = F.parse_all(["abcdef"], bits=16).index_words()
    assert w.nbytes == 8 * 1024
    w, b = F.parse_all(["abcdef"], bits=24).index_words()
    assert w.nbytes == 2 * 1024 * 1024
    assert F.parse_all(["abcdef"]).bits == 16


def test_index_never_loses_a_match(native, oracle):
    # src/filter.rs the_index_never_loses_a_match: constructed keys always match
    F = native.filter.FilterSet
    fs = F.parse_all(["abcd", "abcdef", "zzzz", "qrst", "mnopqr", "a" * 20])
    texts = fs.texts()
    rng = random.Random(1)
    for n in range(4000):
        t = texts[n % len(texts)]
        raw, bits = oracle.base32_decode_bits(t)
        nb = (bits + 7) // 8
        rem = bits % 8
        mask = 0xFF if rem == 0 else (0xFF << (8 - rem)) & 0xFF
        noise = bytes(rng.getrandbits(8) for _ in range(32))
        packed = bytearray(noise)
        packed[: nb - 1] = raw[: nb - 1]
        packed[nb - 1] = (noise[nb - 1] & ~mask & 0xFF) | (raw[nb - 1] & mask)
        assert fs.match_key(bytes(packed)) == texts.index(t)


def test_match_many_agrees_with_match_key(native):
    import numpy as np

    fs = native.filter.FilterSet.parse_all(["abc", "q7", "zz2a"])
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 256, size=(5000, 32), dtype=np.uint8)
    keys[::7, :2] = np.frombuffer(bytes.fromhex("00a1"), dtype=np.uint8)  # 'ab' + bits
    got = fs.match_many(keys)
    want = [fs.match_key(bytes(k)) for k in keys]
    assert [(-1 if w is None else w) for w in want] == got.tolist()


def test_rederivation_against_the_config1_sample(native):
    """The host's independent re-derivation (offset -> secret -> public key)
    gives the reference verifier's full keys, sign bit included, for 1024 of
    config 1's candidates."""
    sample = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config1_sample.json")))
    seed = B(sample["seed"])
    for i, pub in zip(sample["index"], sample["public"]):
        packed = bytearray(B(pub))
        packed[31] &= 0x7F
        pk, _ = native.key.check_hit(seed, 8 * i, bytes(packed))
        assert pk.hex() == pub


def _share(sets, start):
    """Pattern::probability_at (src/filter.rs:443-452) with protocol_allows
    (:226-238): per position, accepted and producible over producible."""
    alphabet = "abcdefghijklmnopqrstuvwxyz234567"
    p = 1.0
    for i, want in enumerate(sets):
        pos = start + i
        room = {alphabet.index("d")} if pos == 55 else {alphabet.index(c) for c in "aiqy"} if pos == 54 else set(range(32))
        p *= len(want & room) / len(room)
    return p


def _either(ps):
    """FilterSet::probability (src/filter.rs:1979-1990): 1 - prod(1 - p)."""
    return -math.expm1(sum(math.log1p(-p) for p in ps))


def test_match_probability(native):
    """og_filters_match_probability restates the reference's FilterSet::
    probability: each kept filter's share with the protocol's tail rooms,
    combined as 1 - prod(1 - p)."""
    from onion_gen_b200 import workloads

    F = native.filter
    alphabet = "abcdefghijklmnopqrstuvwxyz234567"

    def lit(text):
        return [{alphabet.index(c)} for c in text]

    for s in workloads.config4_searches()[:12]:
        kept = []
        for p in sorted(set(s.prefixes)):
            if not (kept and p.startswith(kept[-1])):
                kept.append(p)
        want = _either([_share(lit(p), 0) for p in kept])
        assert math.isclose(F.FilterSet.parse_all(s.prefixes).match_probability(), want, rel_tol=1e-12)
    # a pattern with a wildcard and a class
    want = _either([_share([{alphabet.index("a")}, set(range(32))], 0), _share([{1, 2}, {3}], 0)])
    assert math.isclose(F.FilterSet.parse_all(["a?", "[bc]d"]).match_probability(), want, rel_tol=1e-12)
    # a suffix pays for its tail only where the protocol leaves a choice:
    # 'd' last is free, 'a' before it one in four
    sfx = F.FilterSet.parse_all(["suffix:abcdefgad"])
    assert math.isclose(sfx.match_probability(), 32.0 ** -7 / 4, rel_tol=1e-12)
    assert math.isclose(sfx.match_probability(), _share(lit("abcdefgad"), 56 - 9), rel_tol=1e-12)
    # prefixes and suffixes together
    both = F.FilterSet.parse_all(["ab", "suffix:qqqqqqqid"])
    assert math.isclose(both.match_probability(), _either([32.0 ** -2, 32.0 ** -7 / 4]), rel_tol=1e-12)
