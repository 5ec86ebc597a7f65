"""Prefixes with wildcards and classes (no GPU): the kept set, the bitmap
(BitmapIndex::pattern_slots, src/filter.rs:2480-2530) and the exact match,
against the oracle's restatement."""
import base64

import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import key

ALPHABET = "abcdefghijklmnopqrstuvwxyz234567"

SETS = [
    ["ab?d", "abc", "abce", "x[a-c]z", "ab"],
    ["a?c", "[xyz]2", "k[a-e]?m", "q7", "mm[2-7]"],
    ["?b", "cd"],
    ["[ab][cd][ef][gh]", "zz?zz", "zzz"],
]


@pytest.mark.parametrize("filters", SETS)
@pytest.mark.parametrize("bits", [0, 16, 20])
def test_patterns_against_the_oracle(oracle, filters, bits):
    try:
        fs = F.FilterSet.parse_all(filters, bits=bits)
    except N.OgError:
        # a pattern with more than 4096 slots at this width cannot be indexed
        with pytest.raises(ValueError):
            oracle.FilterSet(filters, bits=bits)
        return
    o = oracle.FilterSet(filters, bits=bits)
    assert fs.texts() == o.canonical()
    words, b = fs.index_words()
    assert b == o.bits and np.array_equal(words, o.words())
    rng = np.random.default_rng(len(filters) + bits)
    keys = rng.integers(0, 256, (20000, 32), dtype=np.uint8)
    # plus keys that start with an instance of each filter
    for i, f in enumerate(filters):
        inst = ""
        j = 0
        while j < len(f):
            if f[j] == "[":
                end = f.index("]", j)
                inst += f[j + 1]
                j = end + 1
            else:
                inst += "a" if f[j] == "?" else f[j]
                j += 1
        text = inst + "".join(rng.choice(list(ALPHABET), 56 - len(inst)))
        keys[i] = np.frombuffer(base64.b32decode(text.upper())[:32], dtype=np.uint8)
    keys[:, 31] &= 0x7F
    got = fs.match_many(keys)
    want = np.array([o.match(bytes(k)) for k in keys], dtype=np.int32)
    assert np.array_equal(got, want)
    assert (got >= 0).any()


def test_pattern_errors():
    with pytest.raises(N.OgError, match="unbalanced"):
        F.FilterSet.parse_all(["ab[c"])
    with pytest.raises(N.OgError, match="fixes no symbol"):
        F.FilterSet.parse_all(["??"])
    with pytest.raises(N.OgError):
        F.FilterSet.parse_all(["????a"])  # 32^3 slots of any index: too broad to index


def test_pattern_full_address_check():
    """A pattern longer than the key-only span (49 symbols) is decided on the
    address."""
    pk = key.public_key(bytes(range(32)))
    addr = key.address(pk)
    pat = addr[:10] + "?" + addr[11:50] + "[" + addr[50] + "a]"
    fs = F.FilterSet.parse_all([pat])
    assert fs.match_address(pk) == 0
    wrong = addr[:10] + "?" + addr[11:50] + ("b" if addr[50] != "b" else "c")
    assert F.FilterSet.parse_all([wrong]).match_address(pk) is None


def test_random_pattern_sets_against_the_oracle(oracle):
    """Seeded random mixes of literals, wildcards and classes: accepted or
    refused alike, the same kept set and bitmap, the same matches."""
    import random

    rng = random.Random(1)

    def sym():
        r = rng.random()
        if r < 0.7:
            return rng.choice(ALPHABET)
        if r < 0.85:
            return "?"
        a, b = sorted(rng.sample(range(32), 2))
        return "[" + (ALPHABET[a] + "-" + ALPHABET[b] if rng.random() < 0.5 else "".join(rng.sample(ALPHABET, 3))) + "]"

    for trial in range(60):
        filters = ["".join(sym() for _ in range(rng.randint(2, 9))) for _ in range(rng.randint(1, 6))]
        bits = rng.choice([0, 16, 20])
        try:
            fs = F.FilterSet.parse_all(filters, bits=bits)
        except N.OgError:
            with pytest.raises(ValueError):
                oracle.FilterSet(filters, bits=bits)
            continue
        o = oracle.FilterSet(filters, bits=bits)
        assert fs.texts() == o.canonical() and fs.bits == o.bits
        assert np.array_equal(fs.index_words()[0], o.words())
        keys = np.random.default_rng(trial).integers(0, 256, (2000, 32), dtype=np.uint8)
        keys[:, 31] &= 0x7F
        want = np.array([o.match(bytes(k)) for k in keys], dtype=np.int32)
        assert np.array_equal(fs.match_many(keys), want)
