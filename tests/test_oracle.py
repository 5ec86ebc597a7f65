"""The CPU oracle pinned to the golden fixtures (no GPU).

The fixtures come from the reference's own Python verifier, hashlib, base64
and big integers (tests/golden/make_golden.py). The oracle is trusted as a
checker only because it passes these.
"""
import json
import os

import numpy as np
import pytest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
B = bytes.fromhex


@pytest.mark.parametrize("case", GOLDEN["field"], ids=lambda c: c["a"][:8])
def test_field_against_big_integers(oracle, case):
    a, b = B(case["a"]), B(case["b"])
    assert oracle.fe_mul(a, b).hex() == case["mul"]
    assert oracle.fe_add(a, b).hex() == case["add"]
    assert oracle.fe_sub(a, b).hex() == case["sub"]
    assert oracle.fe_sq(a).hex() == case["sq"]
    assert oracle.fe_invert(a).hex() == case["inv"]
    assert oracle.fe_canon(a).hex() == case["canon"]


def test_hashes(oracle):
    for h in GOLDEN["hashes"]:
        m = B(h["msg"])
        assert oracle.sha512(m).hex() == h["sha512"]
        assert oracle.sha3_256(m).hex() == h["sha3_256"]


def test_base32(oracle):
    for c in GOLDEN["base32"]:
        assert oracle.base32_encode(B(c["bytes"])) == c["text"]
        dec, bits = oracle.base32_decode_bits(c["text"])
        assert dec[: len(B(c["bytes"]))] == B(c["bytes"])
        assert bits == 5 * len(c["text"])


def test_base32_rejects_bad_symbols_with_position(oracle):
    # src/base32.rs rejects_invalid_character_with_position
    with pytest.raises(ValueError, match="position 2"):
        oracle.base32_decode_bits("ab0cd")
    with pytest.raises(ValueError, match="position 4"):
        oracle.base32_decode_bits("zzzz1")


def test_keys_against_reference_verifier(oracle):
    for k in GOLDEN["keys"]:
        seed = B(k["seed"])
        assert oracle.secret_scalar(seed).hex() == k["scalar"]
        assert oracle.public_key(seed).hex() == k["public"]
        assert oracle.address(B(k["public"])) + ".onion" == k["address"]


def test_address_shape(oracle):
    # src/key.rs address_has_protocol_shape: 56 symbols, ends in d, penultimate in aiqy
    for k in GOLDEN["keys"]:
        a = oracle.address(B(k["public"]))
        assert len(a) == 56 and a.endswith("d") and a[-2] in "aiqy"


def test_chain_numbering_against_reference_verifier(oracle):
    """Element i of BatchEngine from the base point is the key of scalar + 8i."""
    seed = bytes(32)
    start = oracle.scalar_base_mult(oracle.secret_scalar(seed))
    small = [o for o in GOLDEN["offsets"] if o["offset"] < 8 * 70000]
    n = max(o["offset"] for o in small) // 8 + 1
    keys = oracle.chain_keys(start, 256, n, signed=True)
    for o in small:
        i = o["offset"] // 8
        assert keys[32 * i : 32 * i + 32].hex() == o["public"], o["offset"]
    for o in GOLDEN["offsets"]:
        sec = oracle.expanded_secret_at_offset(seed, o["offset"])
        p = oracle.pack(oracle.scalar_base_mult(sec[:32]))
        assert p.hex() == o["public"]


def test_curve_constants(oracle):
    c = GOLDEN["curve"]
    bp = oracle.lib()
    import ctypes

    buf = ctypes.create_string_buffer(128)
    bp.orc_basepoint(buf)
    assert buf.raw[:32].hex() == c["base_x"] and buf.raw[32:64].hex() == c["base_y"]
    assert oracle.check_group_order()
    assert oracle.check_eight_basepoint()
    # 8G from the scalar multiplication agrees with the verifier's 8B
    e8 = oracle.multiple_of_eight_g(1)
    import ctypes as C

    x, y = C.create_string_buffer(32), C.create_string_buffer(32)
    oracle.lib().orc_to_affine(e8, x, y)
    P = 2**255 - 19
    xi, yi = int.from_bytes(x.raw, "little"), int.from_bytes(y.raw, "little")
    assert ((yi + xi) % P).to_bytes(32, "little").hex() == c["eight_ypx"]
    assert ((yi - xi) % P).to_bytes(32, "little").hex() == c["eight_ymx"]


def test_block_seeds(oracle):
    for b in GOLDEN["block_seeds"]:
        assert oracle.block_seed(B(b["root"]), b["index"]).hex() == b["seed"]


def test_scalar_addition_and_clamping(oracle):
    # src/key.rs scalar_addition_is_little_endian, clamping_check_rejects_broken_scalars
    sk = oracle.add_to_scalar(bytes(32), 1)
    assert sk[0] == 1
    v = bytearray(b"\xff" * 32)
    v[1] = 0
    r = oracle.add_to_scalar(bytes(v), 1)
    assert r[0] == 0 and r[1] == 1
    good = oracle.secret_scalar(bytes(32))
    assert oracle.clamping_intact(good)
    for i, mask, setbit in [(0, 1, True), (31, 128, True), (31, 64, False)]:
        b = bytearray(good)
        b[i] = b[i] | mask if setbit else b[i] & ~mask
        assert not oracle.clamping_intact(bytes(b))


def test_offset_breaking_clamping_is_refused(oracle):
    seed = bytes(32)
    sk = oracle.secret_scalar(seed)
    top = (1 << 254) + (1 << 255)  # a delta that carries into bit 254
    room = (1 << 255) - int.from_bytes(sk, "little")
    assert room > 0
    # the largest 64-bit offset cannot reach bit 254, so it stays clamped
    assert oracle.expanded_secret_at_offset(seed, 8 * ((1 << 61) - 1)) is not None
    assert top > 0


def test_batch_size_does_not_change_results(oracle):
    # src/batch.rs batch_size_does_not_change_results (sizes 512, 8192, 3)
    start = oracle.scalar_base_mult(oracle.secret_scalar(bytes(range(32))))
    ref = oracle.chain_keys(start, 512, 1536)
    assert oracle.chain_keys(start, 8192, 1536) == ref
    assert oracle.chain_keys(start, 3, 1536) == ref
    assert oracle.chain_keys_mt(start, 0, 1536, threads=4) == ref


def test_pair_engine_agrees_with_chain_engine(oracle):
    # src/pairs.rs: every candidate is the key at its delta; rounds tile without gaps
    start = oracle.scalar_base_mult(oracle.secret_scalar(bytes(32)))
    for half in (1, 8, 96):
        keys, deltas = oracle.pair_keys(start, half, 3)
        n = 3 * (2 * half + 1)
        assert sorted(int(d) for d in deltas) == [8 * (i + 1) for i in range(n)]
        chain = oracle.chain_keys(start, 64, n + 1)
        for i, d in enumerate(deltas):
            j = int(d) // 8
            assert keys[32 * i : 32 * i + 32] == chain[32 * j : 32 * j + 32]


def test_reference_device_offsets(oracle):
    # src/gpu/cuda.rs:332-354: slot 192 is the centre, even slots +, odd slots -
    threads = 1 << 14
    assert oracle.cuda_offset(0, 192, 0, threads) == 97 * 8
    assert oracle.cuda_offset(0, 0, 0, threads) == 98 * 8
    assert oracle.cuda_offset(0, 1, 0, threads) == 96 * 8
    assert oracle.cuda_offset(0, 191, 0, threads) == 8
    assert oracle.cuda_offset(0, 190, 0, threads) == 193 * 8
    seen = {oracle.cuda_offset(t, s, l, 4) for t in range(4) for s in range(193) for l in range(2)}
    assert seen == {8 * (i + 1) for i in range(4 * 193 * 2)}


def test_reference_hit_room(oracle):
    # src/gpu/mod.rs:306-312
    assert oracle.hit_room(0, 16) == 4096
    assert oracle.hit_room(1 << 40, 16) == 1 << 18
    assert oracle.hit_room(1 << 30, 20) == 4 * 1024 + 1024


SAMPLE = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config1_sample.json")))


def test_config1_sample_against_reference_verifier(oracle):
    """1024 of config 1's 2^20 candidates (seed LE32(0), candidate i = scalar
    + 8 i), computed by the reference's own verifier: the oracle's chain
    engine (src/batch.rs) gives the same keys, sign bit cleared."""
    seed = bytes.fromhex(SAMPLE["seed"])
    start = oracle.scalar_base_mult(oracle.secret_scalar(seed))
    keys = oracle.chain_keys_mt(start, 0, 1 << 20)
    for i, pub in zip(SAMPLE["index"], SAMPLE["public"]):
        want = bytearray(bytes.fromhex(pub))
        want[31] &= 0x7F
        assert keys[32 * i: 32 * i + 32] == bytes(want), i


def test_pair_rate_on_one_search(oracle):
    """The CPU baseline's rate run over one search: a rate and a count for a
    real prefix index; a missing index or a bad width is refused (0)."""
    f = oracle.FilterSet(["cpejtg"])
    r, ex = oracle.pair_rate_search(2, 0.2, 256, bytes(32), f.words(), f.bits)
    assert r > 0 and ex > 0
    r, ex = oracle.pair_rate_search(2, 0.2, 256, bytes(32), f.words(), 0)
    assert r == 0 and ex == 0
