"""Generates the golden fixtures under tests/golden/ (run once, in a container
where the reference project is mounted; the outputs are committed).

Sources, none of them this project's code:
  * the reference's own stdlib-only verifier
    (scripts/verify/verify-onion-address.py: RFC 8032 scalar multiplication
    and the v3 address), imported from the reference tree;
  * Python's hashlib (SHA-512, SHA3-256) and base64 (RFC 4648 base32);
  * Python big integers for GF(2^255-19).

    python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import base64
import hashlib
import importlib.util
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
P = 2**255 - 19


def load_verifier(ref_root):
    path = os.path.join(ref_root, "scripts", "verify", "verify-onion-address.py")
    spec = importlib.util.spec_from_file_location("ref_verify", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def le(n: int) -> str:
    return (n % (1 << 256)).to_bytes(32, "little").hex()


def secret_scalar(seed: bytes) -> bytes:
    d = bytearray(hashlib.sha512(seed).digest()[:32])
    d[0] &= 248
    d[31] &= 63
    d[31] |= 64
    return bytes(d)


def xorshift_seed(n: int) -> bytes:
    """The seed_from(n) helper of the reference's unit tests (src/key.rs:218-230)."""
    out = b""
    x = (n * 0x9E3779B97F4A7C15 + 0x12345678) & ((1 << 64) - 1)
    for _ in range(4):
        x ^= (x << 13) & ((1 << 64) - 1)
        x ^= x >> 7
        x ^= (x << 17) & ((1 << 64) - 1)
        out += x.to_bytes(8, "little")
    return out


def main(ref_root):
    V = load_verifier(ref_root)
    rng = random.Random(20260101)

    # ---- keys: seed -> scalar -> public key -> address ----
    keys = []
    seeds = [i.to_bytes(32, "little") for i in range(24)] + [xorshift_seed(n) for n in range(16)]
    for s in seeds:
        sk = secret_scalar(s)
        pk = V.public_from_secret(sk)
        keys.append({"seed": s.hex(), "scalar": sk.hex(), "public": pk.hex(), "address": V.onion_address(pk)})

    # ---- the chain numbering: candidate i of a base scalar is scalar + 8 i ----
    offsets = []
    s0 = secret_scalar((0).to_bytes(32, "little"))
    base = int.from_bytes(s0, "little")
    for i in [0, 1, 2, 255, 256, 257, 4095, 4096, 65793, (1 << 20) - 1, 12345678, 1 << 32, (1 << 35) + 3]:
        sc = base + 8 * i
        pk = V.public_from_secret(sc.to_bytes(32, "little"))
        packed = bytearray(pk)
        packed[31] &= 0x7F
        offsets.append({"seed": (0).to_bytes(32, "little").hex(), "offset": 8 * i, "public": pk.hex(),
                        "packed": bytes(packed).hex()})

    # ---- field arithmetic ----
    field = []
    edge = [0, 1, 2, 19, P - 1, P, P + 1, 2 * P - 1, 2 * P, (1 << 255) - 1, (1 << 255), (1 << 256) - 1,
            (1 << 256) - 38, (1 << 256) - 39, 38, 37]
    vals = edge + [rng.getrandbits(256) for _ in range(48)] + [rng.getrandbits(255) for _ in range(16)]
    for i, a in enumerate(vals):
        b = vals[(i * 7 + 3) % len(vals)]
        field.append({
            "a": le(a), "b": le(b),
            "mul": le(a * b % P), "add": le((a + b) % P), "sub": le((a - b) % P), "sq": le(a * a % P),
            "inv": le(pow(a % P, P - 2, P)), "canon": le(a % P),
        })

    # ---- curve constants: base point and 8G in cached form (y+x, y-x, 2d x y) ----
    def affine(pt):
        x, y, z, _ = pt
        zi = pow(z, P - 2, P)
        return x * zi % P, y * zi % P

    bx, by = V.BX, V.BY
    ex, ey = affine(V._scalar_mult_base(8))
    two_d = 2 * V.D % P
    curve = {
        "base_x": le(bx), "base_y": le(by), "two_d": le(two_d),
        "eight_ypx": le((ey + ex) % P), "eight_ymx": le((ey - ex) % P), "eight_t2d": le(two_d * ex * ey % P),
        "group_order": le(2**252 + 27742317777372353535851937790883648493),
    }

    # ---- hashes, base32, block seeds ----
    hashes = []
    for n in [0, 1, 3, 32, 55, 56, 64, 111, 112, 127, 128, 135, 136, 137, 200, 271, 272, 500]:
        m = bytes(rng.getrandbits(8) for _ in range(n))
        hashes.append({"msg": m.hex(), "sha512": hashlib.sha512(m).hexdigest(), "sha3_256": hashlib.sha3_256(m).hexdigest()})
    b32 = []
    for n in list(range(1, 11)) + [32, 35]:
        m = bytes(rng.getrandbits(8) for _ in range(n))
        b32.append({"bytes": m.hex(), "text": base64.b32encode(m).decode().rstrip("=").lower()})
    blocks = []
    root = bytes(rng.getrandbits(8) for _ in range(32))
    for idx in [0, 1, 2, 1000, (1 << 40) + 5]:
        d = hashlib.sha512(b"onion-gen block v1" + root + idx.to_bytes(8, "little")).digest()[:32]
        blocks.append({"root": root.hex(), "index": idx, "seed": d.hex()})

    out = {
        "generated_by": "tests/golden/make_golden.py",
        "keys": keys, "offsets": offsets, "field": field, "curve": curve,
        "hashes": hashes, "base32": b32, "block_seeds": blocks,
    }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(keys)} keys, {len(offsets)} offsets, {len(field)} field cases")

    # ---- config 1: a sample of its 2^20 candidates, by the verifier ----
    # candidate i of the base scalar of seed LE32(0) is the key of scalar + 8 i
    srng = random.Random(1)
    idx = sorted(srng.sample(range(1 << 20), 1024))
    pubs = [V.public_from_secret((base + 8 * i).to_bytes(32, "little")).hex() for i in idx]
    with open(os.path.join(HERE, "config1_sample.json"), "w") as f:
        json.dump({"generated_by": "tests/golden/make_golden.py", "seed": (0).to_bytes(32, "little").hex(),
                   "index": idx, "public": pubs}, f)
    print(f"wrote {len(idx)} config-1 keys")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
