"""Keys, offsets and addresses (src/key.rs), through the engine's host code."""
from __future__ import annotations

import ctypes as C

from . import _native as N


def _buf(n):
    return C.create_string_buffer(n)


def seed_from_int(i: int) -> bytes:
    """The 32-byte little-endian encoding of ``i`` — the seeds of the workloads."""
    return int(i).to_bytes(32, "little")


def secret_scalar(seed: bytes) -> bytes:
    out = _buf(32)
    N.lib.og_secret_scalar(bytes(seed), out)
    return out.raw


def expanded_secret_key(seed: bytes) -> bytes:
    out = _buf(64)
    N.lib.og_expanded_secret_key(bytes(seed), out)
    return out.raw


def expanded_secret_at_offset(seed: bytes, offset: int):
    out = _buf(64)
    ok = N.lib.og_expanded_secret_at_offset(bytes(seed), offset, out)
    return out.raw if ok else None


def scalar_base_mult(scalar: bytes) -> bytes:
    out = _buf(128)
    N.lib.og_scalar_base_mult(bytes(scalar), out)
    return out.raw


def start_point(seed: bytes) -> bytes:
    """s * B for the seed's clamped scalar: the point an engine starts from."""
    return scalar_base_mult(secret_scalar(seed))


def pack(point: bytes) -> bytes:
    out = _buf(32)
    N.lib.og_pack(bytes(point), out)
    return out.raw


def public_key(seed: bytes) -> bytes:
    return pack(start_point(seed))


def address(pk: bytes) -> str:
    out = _buf(57)
    N.lib.og_address(bytes(pk), out)
    return out.value.decode()


def hostname(pk: bytes) -> str:
    return address(pk) + ".onion"


def block_seed(root: bytes, index: int) -> bytes:
    out = _buf(32)
    N.lib.og_block_seed(bytes(root), index, out)
    return out.raw


def check_hit(seed: bytes, offset: int, packed: bytes):
    """Re-derives the candidate at ``offset`` (src/run.rs:1089-1104).

    Returns ``(public_key, secret64)`` when the device's packed key is the
    key of that offset; raises ``OgError`` (OG_E_VERIFY) when it is not and
    ``OG_E_ARG`` when the offset broke clamping."""
    pk = _buf(32)
    sk = _buf(64)
    rc = N.lib.og_check_hit(bytes(seed), offset, bytes(packed), pk, sk)
    if rc != N.OG_OK:
        raise N.OgError(rc, f"offset {offset}")
    return pk.raw, sk.raw
