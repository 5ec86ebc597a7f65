// Keccak-f[1600] and the v3 onion address checksum on the device.
//
// The permutation follows FIPS 202 section 3: theta, rho and pi, chi, iota
// over 24 rounds, the round constants from the degree-8 LFSR of 3.2.5 and
// the rotation offsets from the (x, y) -> (y, 2x + 3y) walk of 3.2.2, both
// computed at compile time. The checksum is SHA3-256(".onion checksum" ||
// pk || 0x03)[0..2] (src/key.rs:106-132): one 48-byte message, one block.
#pragma once
#include <cstdint>

namespace og {

struct KeccakConsts {
    uint64_t rc[24];
    uint32_t rot[25];  // index x + 5 y
};

__host__ __device__ constexpr KeccakConsts keccak_consts() {
    KeccakConsts k{};
    uint32_t lfsr = 1;
    for (int r = 0; r < 24; r++) {
        uint64_t c = 0;
        for (int j = 0; j < 7; j++) {
            if (lfsr & 1) c |= 1ULL << ((1u << j) - 1);
            lfsr = ((lfsr << 1) ^ ((lfsr & 0x80) ? 0x71 : 0)) & 0xff;
        }
        k.rc[r] = c;
    }
    k.rot[0] = 0;
    uint32_t x = 1, y = 0;
    for (uint32_t t = 0; t < 24; t++) {
        k.rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
        const uint32_t nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    return k;
}

__device__ __forceinline__ uint64_t rotl64(uint64_t v, uint32_t n) { return n ? (v << n) | (v >> (64 - n)) : v; }

// The round constants, read per round from the constant bank.
static __constant__ KeccakConsts KECCAK_CONSTS = keccak_consts();

__device__ __forceinline__ void keccak_f1600(uint64_t a[25]) {
    constexpr KeccakConsts K = keccak_consts();
#pragma unroll 1
    for (int r = 0; r < 24; r++) {
        uint64_t c[5], b[25];
#pragma unroll
        for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) {
            const uint64_t d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
#pragma unroll
            for (int y = 0; y < 5; y++) a[x + 5 * y] ^= d;
        }
#pragma unroll
        for (int x = 0; x < 5; x++)
#pragma unroll
            for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], K.rot[x + 5 * y]);
#pragma unroll
        for (int y = 0; y < 5; y++)
#pragma unroll
            for (int x = 0; x < 5; x++)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= KECCAK_CONSTS.rc[r];
    }
}

// The two checksum bytes of a full public key given as four little-endian
// 64-bit words (sign bit included), returned as byte0 | byte1 << 8.
__device__ __forceinline__ uint32_t onion_checksum(const uint64_t pk[4]) {
    // ".onion c" and "hecksum", little-endian
    constexpr uint64_t C0 = 0x63206e6f696e6f2eULL;
    constexpr uint64_t C1 = 0x006d75736b636568ULL;
    uint64_t a[25];
#pragma unroll
    for (int i = 0; i < 25; i++) a[i] = 0;
    // message = tag (15 bytes) || pk (32) || 0x03, padded with 0x06 ... 0x80
    a[0] = C0;
    a[1] = C1 | (pk[0] << 56);
    a[2] = (pk[0] >> 8) | (pk[1] << 56);
    a[3] = (pk[1] >> 8) | (pk[2] << 56);
    a[4] = (pk[2] >> 8) | (pk[3] << 56);
    a[5] = (pk[3] >> 8) | (0x03ULL << 56);
    a[6] = 0x06;
    a[16] = 0x80ULL << 56;
    keccak_f1600(a);
    return (uint32_t)(a[0] & 0xffff);
}

}  // namespace og
