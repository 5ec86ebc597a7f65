"""Address filters (src/filter.rs), built by the engine's host code.

``FilterSet.parse_all(["abc", "prefix:def", "suffix:xyz2?[a-c]aad"])`` sorts,
drops absorbed prefixes, builds the prefix bitmap (width chosen as
src/filter.rs:2279-2295 does unless ``bits`` is given) and answers
``match_key`` exactly for the prefixes. ``suffix:`` filters get their own
bitmap keyed on the end of the key-derived span (src/filter.rs:2393-2480) and
are decided on the full address (``match_address``). Other forms raise
``OgError`` (OG_E_FILTER).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class FilterSet:
    def __init__(self, handle):
        self._h = handle

    @classmethod
    def parse_all(cls, filters, bits: int = 0) -> "FilterSet":
        text = "\n".join(filters).encode()
        h = C.c_void_p()
        err = N.errbuf()
        N.check(N.lib.og_filters_new(text, bits, C.byref(h), err, 512), err)
        return cls(h)

    def close(self):
        if getattr(self, "_h", None):
            N.lib.og_filters_free(self._h)
            self._h = None

    __del__ = close

    def __len__(self):
        return N.lib.og_filters_count(self._h)

    def texts(self):
        out = []
        b = C.create_string_buffer(4096)
        for i in range(len(self)):
            N.lib.og_filters_text(self._h, i, b, 4096)
            out.append(b.value.decode())
        return out

    def index_words(self):
        """(words uint64[], bits) — FilterSet::index_words (src/filter.rs:1857)."""
        p = C.POINTER(C.c_uint64)()
        n = N.lib.og_filters_words(self._h, C.byref(p))
        return np.ctypeslib.as_array(p, shape=(n,)).copy(), N.lib.og_filters_bits(self._h)

    @property
    def bits(self) -> int:
        return N.lib.og_filters_bits(self._h)

    def occupancy(self) -> float:
        return N.lib.og_filters_occupancy(self._h)

    def match_probability(self) -> float:
        """The chance that a uniform key matches some filter exactly."""
        return N.lib.og_filters_match_probability(self._h)

    def match_many(self, packed) -> np.ndarray:
        """match_key over an (n, 32) uint8 array: int32 indices, -1 where none matches."""
        arr = np.ascontiguousarray(packed, dtype=np.uint8)
        out = np.empty(len(arr), dtype=np.int32)
        if len(arr):
            N.lib.og_filters_match_many(self._h, arr.ctypes.data, len(arr), arr.strides[0], out.ctypes.data)
        return out

    def match_key(self, packed: bytes):
        """Index of the filter this packed key matches, or None."""
        i = N.lib.og_filters_match(self._h, bytes(packed))
        return None if i < 0 else i

    def prefix_count(self) -> int:
        """Kept prefixes; filter indices at and above it are suffixes."""
        return N.lib.og_filters_prefix_count(self._h)

    def suffix_index_words(self):
        """(words uint64[], bits) of the suffix bitmap; (empty, 0) without suffixes."""
        p = C.POINTER(C.c_uint64)()
        n = N.lib.og_filters_suffix_words(self._h, C.byref(p))
        if n == 0:
            return np.zeros(0, dtype=np.uint64), 0
        return np.ctypeslib.as_array(p, shape=(n,)).copy(), N.lib.og_filters_suffix_bits(self._h)

    def match_address(self, pk: bytes):
        """The full check of a public key (sign bit included) on its address:
        the index of the first filter it matches, or None."""
        i = N.lib.og_filters_match_address(self._h, bytes(pk))
        return None if i < 0 else i
