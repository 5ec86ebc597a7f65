"""Suffix filters on the host (no GPU): parsing, the suffix bitmap and the
full-address match, against the oracle's restatement of src/filter.rs and
against the reference's own tests of the `suffix:` form
(rejects_unreachable_suffixes, the_suffix_bitmap_never_rules_out_a_reachable_suffix,
the_key_decides_the_part_of_a_suffix_that_reaches_it)."""
import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import key

ALPHABET = "abcdefghijklmnopqrstuvwxyz234567"


def test_unreachable_tails_are_rejected():
    with pytest.raises(N.OgError, match="always 'd'"):
        F.FilterSet.parse_all(["suffix:abc"])
    with pytest.raises(N.OgError, match="second-to-last"):
        F.FilterSet.parse_all(["suffix:abd"])
    # reachable, but too short to index: refused by the bitmap, not the parser
    for good in ["suffix:d", "suffix:ad", "suffix:id", "suffix:qd", "suffix:yd"]:
        with pytest.raises(N.OgError, match="reaches too little"):
            F.FilterSet.parse_all([good])
    for bad, what in [("suffix:a[bc", "unbalanced"), ("suffix:ab]d", "unbalanced"), ("suffix:[c-a]ad", "empty range"),
                      ("suffix:??", "fixes no symbol"), ("suffix:a1ad", "invalid character")]:
        with pytest.raises(N.OgError, match=what):
            F.FilterSet.parse_all([bad])


@pytest.mark.parametrize(
    "bodies",
    [
        ["aaaaaaaazad"],
        ["xyz2?[a-c]aad", "aaaaaaaazad"],
        [f"{ALPHABET[i % 32]}{ALPHABET[(i * 7) % 32]}[a-f]?{ALPHABET[(i * 3) % 32]}ab2{ALPHABET[i % 5]}qd" for i in range(60)],
        ["bcdefgh[q-t]ad", "zzzzzzzzzzzzid"],
        ["mmmmmmmm?yd", "mmmmmmmm?yd"],
    ],
)
def test_suffix_bitmap_equals_the_oracle(oracle, bodies):
    """Same suffixes kept, same width chosen, same words."""
    fs = F.FilterSet.parse_all(["suffix:" + b for b in bodies])
    words, b = fs.suffix_index_words()
    o = oracle.SuffixSet(bodies)
    assert b == o.bits and len(fs) == len(o)
    assert np.array_equal(words, o.words())
    assert fs.prefix_count() == 0 and fs.bits == 0


def xorshift_keys(n, state=0x2545F4914F6CDD1D):
    out = np.zeros((n, 32), dtype=np.uint8)
    m = (1 << 64) - 1
    for i in range(n):
        row = bytearray()
        for _ in range(4):
            state ^= (state << 13) & m
            state ^= state >> 7
            state ^= (state << 17) & m
            row += state.to_bytes(8, "little")
        out[i] = np.frombuffer(bytes(row), dtype=np.uint8)
    return out


def slot_of(packed, bits):
    """The suffix bitmap slot: base32 bits [255 - bits, 255) of the key."""
    w = 0
    for b in packed[24:32]:
        w = (w << 8) | int(b)
    return (w >> 1) & ((1 << bits) - 1)


def test_the_suffix_bitmap_never_rules_out_a_reachable_suffix(oracle):
    # the reference's own case: forty eight-symbol suffixes, three symbols of
    # each inside the key
    bodies = ["".join(ALPHABET[(i * 5 + j * 7) % 32] for j in range(6)) + "ad" for i in range(40)]
    fs = F.FilterSet.parse_all(["suffix:" + b for b in bodies])
    words, bits = fs.suffix_index_words()
    o = oracle.SuffixSet(bodies)
    alive = 0
    for packed in xorshift_keys(20000):
        p = bytes(packed)
        naive = any(o.key_prefilter(i, p) for i in range(len(o)))
        s = slot_of(packed, bits)
        ours = bool((int(words[s >> 6]) >> (s & 63)) & 1)
        assert ours == o.may_match(p)
        assert not naive or ours
        alive += naive
    assert alive > 0


def test_the_key_decides_the_part_of_a_suffix_that_reaches_it(oracle):
    o = oracle.SuffixSet(["aaaaaaaazad"])
    hits = 0
    for n in range(64):
        packed = bytearray(32)
        packed[20] = n
        packed[28] = (n * 7) & 0xFF
        hits += o.key_prefilter(0, bytes(packed))
    assert hits < 64


def test_full_address_match_equals_the_oracle(oracle):
    rng = np.random.default_rng(5)
    pks = []
    for i in range(64):
        seed = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
        pks.append(key.public_key(seed))
    # suffixes taken from real addresses (with their sign and checksum), one
    # with the sign bit of symbol 49 flipped, plus a literal prefix
    a0, a1 = key.address(pks[0]), key.address(pks[1])
    flipped = a1[46:49] + ALPHABET[ALPHABET.index(a1[49]) ^ 2] + a1[50:56]
    filters = ["suffix:" + a0[46:], "suffix:" + a1[44:], "suffix:" + flipped, a1[:3]]
    fs = F.FilterSet.parse_all(filters)
    o = oracle.SuffixSet([a0[46:], a1[44:], flipped])
    np_ = fs.prefix_count()
    texts = fs.texts()
    for pk in pks:
        m = fs.match_address(pk)
        addr = key.address(pk)
        if m is not None and m < np_:
            assert addr.startswith(texts[m])
            continue
        j = o.match_pk(pk)
        assert (m is None) == (j < 0)
        if m is not None:
            assert texts[m] == "suffix:" + addr[56 - len(texts[m]) + 7:]
    assert fs.match_address(pks[0]) is not None
    assert texts[fs.match_address(pks[1])] in ("suffix:" + a1[44:], a1[:3])
