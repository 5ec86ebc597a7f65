#include "hash.h"

#include <cstring>

namespace og {

namespace {

// FIPS 180-4 4.2.3: first 64 bits of the fractional parts of the cube roots
// of the first eighty primes.
const uint64_t K512[80] = {
    0x428a2f98d728ae22ULL, 0x7137449123ef65cdULL, 0xb5c0fbcfec4d3b2fULL, 0xe9b5dba58189dbbcULL,
    0x3956c25bf348b538ULL, 0x59f111f1b605d019ULL, 0x923f82a4af194f9bULL, 0xab1c5ed5da6d8118ULL,
    0xd807aa98a3030242ULL, 0x12835b0145706fbeULL, 0x243185be4ee4b28cULL, 0x550c7dc3d5ffb4e2ULL,
    0x72be5d74f27b896fULL, 0x80deb1fe3b1696b1ULL, 0x9bdc06a725c71235ULL, 0xc19bf174cf692694ULL,
    0xe49b69c19ef14ad2ULL, 0xefbe4786384f25e3ULL, 0x0fc19dc68b8cd5b5ULL, 0x240ca1cc77ac9c65ULL,
    0x2de92c6f592b0275ULL, 0x4a7484aa6ea6e483ULL, 0x5cb0a9dcbd41fbd4ULL, 0x76f988da831153b5ULL,
    0x983e5152ee66dfabULL, 0xa831c66d2db43210ULL, 0xb00327c898fb213fULL, 0xbf597fc7beef0ee4ULL,
    0xc6e00bf33da88fc2ULL, 0xd5a79147930aa725ULL, 0x06ca6351e003826fULL, 0x142929670a0e6e70ULL,
    0x27b70a8546d22ffcULL, 0x2e1b21385c26c926ULL, 0x4d2c6dfc5ac42aedULL, 0x53380d139d95b3dfULL,
    0x650a73548baf63deULL, 0x766a0abb3c77b2a8ULL, 0x81c2c92e47edaee6ULL, 0x92722c851482353bULL,
    0xa2bfe8a14cf10364ULL, 0xa81a664bbc423001ULL, 0xc24b8b70d0f89791ULL, 0xc76c51a30654be30ULL,
    0xd192e819d6ef5218ULL, 0xd69906245565a910ULL, 0xf40e35855771202aULL, 0x106aa07032bbd1b8ULL,
    0x19a4c116b8d2d0c8ULL, 0x1e376c085141ab53ULL, 0x2748774cdf8eeb99ULL, 0x34b0bcb5e19b48a8ULL,
    0x391c0cb3c5c95a63ULL, 0x4ed8aa4ae3418acbULL, 0x5b9cca4f7763e373ULL, 0x682e6ff3d6b2b8a3ULL,
    0x748f82ee5defb2fcULL, 0x78a5636f43172f60ULL, 0x84c87814a1f0ab72ULL, 0x8cc702081a6439ecULL,
    0x90befffa23631e28ULL, 0xa4506cebde82bde9ULL, 0xbef9a3f7b2c67915ULL, 0xc67178f2e372532bULL,
    0xca273eceea26619cULL, 0xd186b8c721c0c207ULL, 0xeada7dd6cde0eb1eULL, 0xf57d4f7fee6ed178ULL,
    0x06f067aa72176fbaULL, 0x0a637dc5a2c898a6ULL, 0x113f9804bef90daeULL, 0x1b710b35131c471bULL,
    0x28db77f523047d84ULL, 0x32caab7b40c72493ULL, 0x3c9ebe0a15c9bebcULL, 0x431d67c49c100d4cULL,
    0x4cc5d4becb3e42b6ULL, 0x597f299cfc657e2aULL, 0x5fcb6fab3ad6faecULL, 0x6c44198c4a475817ULL,
};

// FIPS 180-4 5.3.5: the same for the square roots of the first eight primes.
const uint64_t IV512[8] = {
    0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL, 0xa54ff53a5f1d36f1ULL,
    0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL, 0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL,
};

inline uint64_t rotr(uint64_t x, unsigned n) { return (x >> n) | (x << (64 - n)); }

inline uint64_t load_be64(const uint8_t* p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
    return v;
}

}  // namespace

Sha512::Sha512() { std::memcpy(h_, IV512, sizeof h_); }

void Sha512::block(const uint8_t* p) {
    uint64_t w[80];
    for (int t = 0; t < 16; t++) w[t] = load_be64(p + 8 * t);
    for (int t = 16; t < 80; t++) {
        const uint64_t x = w[t - 15], y = w[t - 2];
        w[t] = (rotr(y, 19) ^ rotr(y, 61) ^ (y >> 6)) + w[t - 7] + (rotr(x, 1) ^ rotr(x, 8) ^ (x >> 7)) +
               w[t - 16];
    }
    uint64_t s[8];
    std::memcpy(s, h_, sizeof s);
    for (int t = 0; t < 80; t++) {
        const uint64_t e = s[4], a = s[0];
        const uint64_t t1 = s[7] + (rotr(e, 14) ^ rotr(e, 18) ^ rotr(e, 41)) + ((e & s[5]) ^ (~e & s[6])) +
                            K512[t] + w[t];
        const uint64_t t2 = (rotr(a, 28) ^ rotr(a, 34) ^ rotr(a, 39)) + ((a & s[1]) ^ (a & s[2]) ^ (s[1] & s[2]));
        for (int i = 7; i > 0; i--) s[i] = s[i - 1];
        s[4] += t1;
        s[0] = t1 + t2;
    }
    for (int i = 0; i < 8; i++) h_[i] += s[i];
}

void Sha512::update(const void* data, size_t len) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    total_ += len;
    while (len) {
        const size_t take = (128 - fill_) < len ? (128 - fill_) : len;
        std::memcpy(buf_ + fill_, p, take);
        fill_ += take;
        p += take;
        len -= take;
        if (fill_ == 128) {
            block(buf_);
            fill_ = 0;
        }
    }
}

void Sha512::finish(uint8_t out[64]) {
    const uint64_t bits = total_ * 8;
    const uint8_t one = 0x80;
    update(&one, 1);
    const uint8_t zero = 0;
    while (fill_ != 112) update(&zero, 1);
    uint8_t len[16] = {0};
    for (int i = 0; i < 8; i++) len[15 - i] = (uint8_t)(bits >> (8 * i));
    update(len, 16);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) out[8 * i + j] = (uint8_t)(h_[i] >> (56 - 8 * j));
}

void sha512(const void* data, size_t len, uint8_t out[64]) {
    Sha512 h;
    h.update(data, len);
    h.finish(out);
}

namespace {

struct KeccakTables {
    uint64_t rc[24];
    unsigned rot[5][5];
    KeccakTables() {
        // Round constants from the degree-8 LFSR of FIPS 202 3.2.5.
        uint8_t lfsr = 1;
        for (int r = 0; r < 24; r++) {
            uint64_t c = 0;
            for (int j = 0; j < 7; j++) {
                if (lfsr & 1) c |= 1ULL << ((1u << j) - 1);
                lfsr = (uint8_t)((lfsr << 1) ^ ((lfsr & 0x80) ? 0x71 : 0));
            }
            rc[r] = c;
        }
        // Rotation offsets from the (x, y) -> (y, 2x + 3y) walk of 3.2.2.
        rot[0][0] = 0;
        unsigned x = 1, y = 0;
        for (unsigned t = 0; t < 24; t++) {
            rot[x][y] = ((t + 1) * (t + 2) / 2) % 64;
            const unsigned nx = y, ny = (2 * x + 3 * y) % 5;
            x = nx;
            y = ny;
        }
    }
};

const KeccakTables& keccak_tables() {
    static const KeccakTables t;
    return t;
}

inline uint64_t rotl(uint64_t v, unsigned n) { return n ? (v << n) | (v >> (64 - n)) : v; }

void keccak_permute(uint64_t st[5][5]) {
    const KeccakTables& T = keccak_tables();
    for (int r = 0; r < 24; r++) {
        uint64_t c[5];
        for (int x = 0; x < 5; x++) c[x] = st[x][0] ^ st[x][1] ^ st[x][2] ^ st[x][3] ^ st[x][4];
        for (int x = 0; x < 5; x++) {
            const uint64_t d = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
            for (int y = 0; y < 5; y++) st[x][y] ^= d;
        }
        uint64_t b[5][5];
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) b[y][(2 * x + 3 * y) % 5] = rotl(st[x][y], T.rot[x][y]);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) st[x][y] = b[x][y] ^ (~b[(x + 1) % 5][y] & b[(x + 2) % 5][y]);
        st[0][0] ^= T.rc[r];
    }
}

}  // namespace

void sha3_256(const void* data, size_t len, uint8_t out[32]) {
    const size_t rate = 136;
    uint64_t st[5][5] = {};
    const uint8_t* p = static_cast<const uint8_t*>(data);
    uint8_t block[136];
    bool done = false;
    while (!done) {
        const size_t take = len < rate ? len : rate;
        std::memset(block, 0, rate);
        std::memcpy(block, p, take);
        if (take < rate) {
            block[take] ^= 0x06;
            block[rate - 1] ^= 0x80;
            done = true;
        }
        for (size_t i = 0; i < rate / 8; i++) {
            uint64_t v = 0;
            for (int j = 7; j >= 0; j--) v = (v << 8) | block[8 * i + j];
            st[i % 5][i / 5] ^= v;
        }
        keccak_permute(st);
        p += take;
        len -= take;
    }
    for (int i = 0; i < 32; i++) out[i] = (uint8_t)(st[(i / 8) % 5][(i / 8) / 5] >> (8 * (i % 8)));
}

}  // namespace og
