// The device half of the suffix filters: a survivor's full key recomputed
// from its scalar offset, its v3 address tail (sign bit, SHA3-256 checksum,
// version) and the exact match against every suffix (FilterSet::match_address,
// src/filter.rs:2152, on the 35 address bytes of src/key.rs:106-132).
#pragma once
#include "keccak.cuh"
#include "search_common.cuh"

namespace og {

// The suffixes of one filter set, and the table of 2^j 8G (j < 64, cached
// form, (j * 3 + {ypx,ymx,t2d}) * 2 + q) the key recomputation walks.
struct SuffixTables {
    const uint32_t* suffixes;  // per suffix MAX_SUFFIX_SYMBOLS + 1 words: its length, then a set per position
    uint32_t nsuffix;
    const uint4* pow8;
};

// Index of the first suffix the key at scalar offset 8 k from `start`
// matches, or 0xffffffff. The key is start + k 8G over the binary expansion
// of k, made affine; its y must equal the survivor's canonical `yrec` (a
// mismatch sets `mismatch` and never matches; the caller counts it). The
// sign bit is the parity of the canonical x.
__device__ __forceinline__ uint32_t suffix_match(const SuffixTables& t, const FeWords& sx, const FeWords& sy,
                                                 const FeWords& sz, const FeWords& st, uint64_t k,
                                                 const uint32_t yrec[8], bool& mismatch) {
    fe X = words_fe(sx), Y = words_fe(sy), Z = words_fe(sz), T = words_fe(st);
#pragma unroll 1
    for (uint32_t j = 0; j < 64; j++)
        if ((k >> j) & 1) {
            const uint4* p = t.pow8 + (size_t)j * 6;
            add_cached(X, Y, Z, T, load_fe(p + 0, 1), load_fe(p + 2, 1), load_fe(p + 4, 1));
        }
    const fe zi = fe_invert(Z);
    const fe x = fe_canon(fe_mulv(X, zi)), y = fe_canon(fe_mulv(Y, zi));
    bool same = true;
#pragma unroll
    for (int q = 0; q < 8; q++) same &= y.v[q] == yrec[q];
    mismatch = !same;
    if (!same) return 0xffffffffu;
    uint64_t pk[4];
#pragma unroll
    for (int q = 0; q < 4; q++) pk[q] = (uint64_t)y.v[2 * q] | ((uint64_t)y.v[2 * q + 1] << 32);
    pk[3] |= (uint64_t)(x.v[0] & 1u) << 63;  // the sign bit
    const uint32_t cs = onion_checksum(pk);
    // pk || checksum || 0x03, and its base32 symbols (five bits each, most
    // significant first)
    uint8_t addr[36];
#pragma unroll
    for (int q = 0; q < 32; q++) addr[q] = (uint8_t)(pk[q / 8] >> (8 * (q % 8)));
    addr[32] = (uint8_t)cs;
    addr[33] = (uint8_t)(cs >> 8);
    addr[34] = 0x03;
    addr[35] = 0;
    for (uint32_t j = 0; j < t.nsuffix; j++) {
        const uint32_t* s = t.suffixes + (size_t)j * (MAX_SUFFIX_SYMBOLS + 1);
        const uint32_t len = s[0], start = MAX_SUFFIX_SYMBOLS - len;
        bool ok = true;
        for (uint32_t i = 0; i < len && ok; i++) {
            const uint32_t bit = (start + i) * 5, byte = bit / 8;
            const uint32_t sym = ((((uint32_t)addr[byte] << 8) | addr[byte + 1]) >> (11 - bit % 8)) & 31u;
            ok = (s[1 + i] >> sym) & 1u;
        }
        if (ok) return j;
    }
    return 0xffffffffu;
}

}  // namespace og
