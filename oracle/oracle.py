"""ctypes front of the CPU oracle (TEST INFRASTRUCTURE).

Loads ``oracle/_build/liboracle.so``, the plain-C restatement of onion-gen's
CPU algorithms. Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module, and only as the checker or as the
timed CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> str:
    """Compiles the oracle with its Makefile when the library is missing or stale."""
    src = os.path.join(HERE, "oracle.c")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P, U8P, SZ, U64, U32 = C.c_void_p, C.c_char_p, C.c_size_t, C.c_uint64, C.c_uint32
        L.orc_pair_rate.restype = C.c_double
        L.orc_pair_rate.argtypes = [C.c_int, C.c_double, SZ, C.POINTER(U64)]
        L.orc_pair_rate_search.restype = C.c_double
        L.orc_pair_rate_search.argtypes = [C.c_int, C.c_double, SZ, C.c_char_p, C.c_void_p, C.c_uint32,
                                           C.POINTER(U64)]
        L.orc_chain_rate.restype = C.c_double
        L.orc_chain_rate.argtypes = [C.c_int, C.c_double, SZ, C.POINTER(U64)]
        L.orc_fset_new.restype = P
        L.orc_fset_new.argtypes = [U8P, U32, U8P, SZ]
        L.orc_fset_free.argtypes = [P]
        L.orc_fset_count.restype = SZ
        L.orc_fset_count.argtypes = [P]
        L.orc_fset_canonical.argtypes = [P, SZ, U8P, SZ]
        L.orc_fset_bits.restype = U32
        L.orc_fset_bits.argtypes = [P]
        L.orc_fset_nwords.restype = SZ
        L.orc_fset_nwords.argtypes = [P]
        L.orc_fset_words.restype = C.POINTER(U64)
        L.orc_fset_words.argtypes = [P]
        L.orc_fset_occupancy.restype = C.c_double
        L.orc_fset_occupancy.argtypes = [P]
        L.orc_fset_may_match.restype = C.c_int
        L.orc_fset_may_match.argtypes = [P, U8P]
        L.orc_fset_match.restype = C.c_long
        L.orc_fset_match.argtypes = [P, U8P]
        L.orc_sset_new.restype = P
        L.orc_sset_new.argtypes = [U8P, U32, U8P, SZ]
        L.orc_sset_free.argtypes = [P]
        L.orc_sset_count.restype = SZ
        L.orc_sset_count.argtypes = [P]
        L.orc_sset_bits.restype = U32
        L.orc_sset_bits.argtypes = [P]
        L.orc_sset_nwords.restype = SZ
        L.orc_sset_nwords.argtypes = [P]
        L.orc_sset_words.restype = C.POINTER(U64)
        L.orc_sset_words.argtypes = [P]
        L.orc_sset_may_match.restype = C.c_int
        L.orc_sset_may_match.argtypes = [P, U8P]
        L.orc_sset_key_prefilter.restype = C.c_int
        L.orc_sset_key_prefilter.argtypes = [P, SZ, U8P]
        L.orc_sset_match_pk.restype = C.c_long
        L.orc_sset_match_pk.argtypes = [P, U8P]
        L.orc_cuda_offset.restype = U64
        L.orc_cuda_offset.argtypes = [U64, U64, U64, U32, U32]
        L.orc_hit_room.restype = U32
        L.orc_hit_room.argtypes = [U64, U32]
        L.orc_expanded_secret_at_offset.restype = C.c_int
        L.orc_expanded_secret_at_offset.argtypes = [U8P, U64, U8P]
        L.orc_add_to_scalar.argtypes = [U8P, U64]
        L.orc_clamping_intact.restype = C.c_int
        L.orc_base32_encode.restype = SZ
        L.orc_base32_decode_bits.restype = C.c_long
        L.orc_base32_decode_bits.argtypes = [U8P, U8P, SZ, C.POINTER(SZ)]
        L.orc_block_seed.argtypes = [U8P, U64, U8P]
        L.orc_multiple_of_eight_g.argtypes = [U64, U8P]
        L.orc_chain_keys.argtypes = [U8P, SZ, SZ, U8P, U8P]
        L.orc_chain_keys_signed.argtypes = [U8P, SZ, SZ, U8P]
        L.orc_chain_keys_mt.argtypes = [U8P, U64, SZ, U8P, C.c_int]
        L.orc_pair_keys.argtypes = [U8P, SZ, SZ, U8P, C.c_void_p]
        L.orc_sha512.argtypes = [U8P, SZ, U8P]
        L.orc_sha3_256.argtypes = [U8P, SZ, U8P]
        L.orc_check_group_order.restype = C.c_int
        L.orc_check_eight_basepoint.restype = C.c_int
        _lib = L
    return _lib


def _buf(n):
    return C.create_string_buffer(n)


def _fe2(fn, a: bytes, b: bytes) -> bytes:
    out = _buf(32)
    fn(a, b, out)
    return out.raw


def fe_mul(a: bytes, b: bytes) -> bytes:
    return _fe2(lib().orc_fe_mul, a, b)


def fe_add(a: bytes, b: bytes) -> bytes:
    return _fe2(lib().orc_fe_add, a, b)


def fe_sub(a: bytes, b: bytes) -> bytes:
    return _fe2(lib().orc_fe_sub, a, b)


def fe_sq(a: bytes) -> bytes:
    out = _buf(32)
    lib().orc_fe_sq(a, out)
    return out.raw


def fe_invert(a: bytes) -> bytes:
    out = _buf(32)
    lib().orc_fe_invert(a, out)
    return out.raw


def fe_canon(a: bytes) -> bytes:
    out = _buf(32)
    lib().orc_fe_canon(a, out)
    return out.raw


def sha512(m: bytes) -> bytes:
    out = _buf(64)
    lib().orc_sha512(m, len(m), out)
    return out.raw


def sha3_256(m: bytes) -> bytes:
    out = _buf(32)
    lib().orc_sha3_256(m, len(m), out)
    return out.raw


def secret_scalar(seed: bytes) -> bytes:
    out = _buf(32)
    lib().orc_secret_scalar(seed, out)
    return out.raw


def expanded_secret_key(seed: bytes) -> bytes:
    out = _buf(64)
    lib().orc_expanded_secret_key(seed, out)
    return out.raw


def expanded_secret_at_offset(seed: bytes, offset: int):
    out = _buf(64)
    ok = lib().orc_expanded_secret_at_offset(seed, offset, out)
    return out.raw if ok else None


def add_to_scalar(sk: bytes, delta: int) -> bytes:
    b = C.create_string_buffer(bytes(sk), 32)
    lib().orc_add_to_scalar(b, delta)
    return b.raw


def clamping_intact(sk: bytes) -> bool:
    return bool(lib().orc_clamping_intact(sk))


def scalar_base_mult(scalar: bytes) -> bytes:
    out = _buf(128)
    lib().orc_scalar_base_mult(scalar, out)
    return out.raw


def point_add(p: bytes, q: bytes) -> bytes:
    out = _buf(128)
    lib().orc_point_add(p, q, out)
    return out.raw


def multiple_of_eight_g(k: int) -> bytes:
    out = _buf(128)
    lib().orc_multiple_of_eight_g(k, out)
    return out.raw


def pack(point: bytes) -> bytes:
    out = _buf(32)
    lib().orc_pack(point, out)
    return out.raw


def public_key(seed: bytes) -> bytes:
    out = _buf(32)
    lib().orc_public_key(seed, out)
    return out.raw


def checksum(pk: bytes) -> bytes:
    out = _buf(2)
    lib().orc_checksum(pk, out)
    return out.raw


def address(pk: bytes) -> str:
    out = _buf(57)
    lib().orc_address(pk, out)
    return out.value.decode()


def block_seed(root: bytes, index: int) -> bytes:
    out = _buf(32)
    lib().orc_block_seed(root, index, out)
    return out.raw


def base32_encode(b: bytes) -> str:
    out = _buf(len(b) * 8 // 5 + 2)
    lib().orc_base32_encode(b, len(b), out)
    return out.value.decode()


def base32_decode_bits(s: str):
    out = _buf(len(s) + 8)
    bits = C.c_size_t()
    n = lib().orc_base32_decode_bits(s.encode(), out, len(s) + 8, C.byref(bits))
    if n < 0:
        raise ValueError(f"invalid symbol at position {-n - 1}")
    return out.raw[:n], bits.value


def chain_keys(start: bytes, batch: int, count: int, signed: bool = False) -> bytes:
    """BatchEngine keys (sign clear unless ``signed``), element i = start + 8i."""
    out = _buf(32 * count)
    if signed:
        lib().orc_chain_keys_signed(start, batch, count, out)
    else:
        lib().orc_chain_keys(start, batch, count, out, None)
    return out.raw


def chain_keys_mt(start: bytes, first: int, count: int, threads: int = 0) -> bytes:
    """Chain keys for elements first .. first+count-1, on several threads."""
    out = _buf(32 * count)
    lib().orc_chain_keys_mt(start, first, count, out, threads or (os.cpu_count() or 1))
    return out.raw


def pair_keys(start: bytes, half: int, rounds: int):
    import numpy as np

    n = (2 * half + 1) * rounds
    keys = _buf(32 * n)
    deltas = np.zeros(n, dtype=np.uint64)
    lib().orc_pair_keys(start, half, rounds, keys, deltas.ctypes.data)
    return keys.raw, deltas


def pair_rate(threads: int, seconds: float, half: int = 96):
    ex = C.c_uint64()
    r = lib().orc_pair_rate(threads, seconds, half, C.byref(ex))
    return r, ex.value


def pair_rate_search(threads: int, seconds: float, half: int, seed: bytes, words, bits: int):
    """pair_rate on one search: the seed's scalar, thread t 2^40 t candidates
    into it, every candidate probed in the search's prefix index."""
    import numpy as np

    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint64))
    ex = C.c_uint64()
    r = lib().orc_pair_rate_search(threads, seconds, half, bytes(seed), w.ctypes.data, bits, C.byref(ex))
    return r, ex.value


def chain_rate(threads: int, seconds: float, batch: int = 8192):
    ex = C.c_uint64()
    r = lib().orc_chain_rate(threads, seconds, batch, C.byref(ex))
    return r, ex.value


def cuda_offset(tid: int, slot: int, launch: int, threads: int, half: int = 96) -> int:
    return lib().orc_cuda_offset(tid, slot, launch, threads, half)


def hit_room(batch: int, bits: int) -> int:
    return lib().orc_hit_room(batch, bits)


def check_group_order() -> bool:
    return bool(lib().orc_check_group_order())


def check_eight_basepoint() -> bool:
    return bool(lib().orc_check_eight_basepoint())


class FilterSet:
    """Literal-prefix FilterSet (sorted, absorbed, bitmap-indexed)."""

    def __init__(self, filters, bits: int = 0):
        err = _buf(256)
        text = "\n".join(filters).encode()
        self._h = lib().orc_fset_new(text, bits, err, 256)
        if not self._h:
            raise ValueError(err.value.decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_fset_free(h)
            self._h = None

    def __len__(self):
        return lib().orc_fset_count(self._h)

    def canonical(self):
        out = []
        b = _buf(4096)
        for i in range(len(self)):
            lib().orc_fset_canonical(self._h, i, b, 4096)
            out.append(b.value.decode())
        return out

    @property
    def bits(self) -> int:
        return lib().orc_fset_bits(self._h)

    def words(self):
        import numpy as np

        n = lib().orc_fset_nwords(self._h)
        p = lib().orc_fset_words(self._h)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def occupancy(self) -> float:
        return lib().orc_fset_occupancy(self._h)

    def may_match(self, packed: bytes) -> bool:
        return bool(lib().orc_fset_may_match(self._h, packed))

    def match(self, packed: bytes) -> int:
        return lib().orc_fset_match(self._h, packed)


class SuffixSet:
    """Suffix filters (the `suffix:` form) with their suffix bitmap."""

    def __init__(self, bodies, bits: int = 0):
        err = _buf(256)
        text = "\n".join(bodies).encode()
        self._h = lib().orc_sset_new(text, bits, err, 256)
        if not self._h:
            raise ValueError(err.value.decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_sset_free(h)
            self._h = None

    def __len__(self):
        return lib().orc_sset_count(self._h)

    @property
    def bits(self) -> int:
        return lib().orc_sset_bits(self._h)

    def words(self):
        import numpy as np

        n = lib().orc_sset_nwords(self._h)
        p = lib().orc_sset_words(self._h)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def may_match(self, packed: bytes) -> bool:
        return bool(lib().orc_sset_may_match(self._h, packed))

    def key_prefilter(self, i: int, packed: bytes) -> bool:
        return bool(lib().orc_sset_key_prefilter(self._h, i, packed))

    def match_pk(self, pk: bytes) -> int:
        return lib().orc_sset_match_pk(self._h, pk)
