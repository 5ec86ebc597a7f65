#include "keys.h"

#include <cstring>

#include "hash.h"

namespace og {

const char BASE32_ALPHABET[33] = "abcdefghijklmnopqrstuvwxyz234567";

int base32_value(char c) {
    if (c >= 'a' && c <= 'z') return c - 'a';
    if (c >= 'A' && c <= 'Z') return c - 'A';
    if (c >= '2' && c <= '7') return c - '2' + 26;
    return -1;
}

// Five bits at a time from the front, the tail padded with zero bits
// (src/base32.rs:42-60).
std::string base32_encode(const uint8_t* bytes, size_t n) {
    std::string out;
    out.reserve((n * 8 + 4) / 5);
    const size_t total = n * 8;
    for (size_t bit = 0; bit < total; bit += 5) {
        unsigned v = 0;
        for (unsigned k = 0; k < 5; k++) {
            const size_t b = bit + k;
            v <<= 1;
            if (b < total) v |= (bytes[b / 8] >> (7 - b % 8)) & 1;
        }
        out.push_back(BASE32_ALPHABET[v]);
    }
    return out;
}

void clamp_scalar(uint8_t sk[32]) {
    sk[0] &= 248;
    sk[31] &= 63;
    sk[31] |= 64;
}

void secret_scalar(const uint8_t seed[32], uint8_t sk[32]) {
    uint8_t d[64];
    sha512(seed, 32, d);
    std::memcpy(sk, d, 32);
    clamp_scalar(sk);
}

void expanded_secret_key(const uint8_t seed[32], uint8_t out[64]) {
    sha512(seed, 32, out);
    clamp_scalar(out);
}

void add_to_scalar(uint8_t sk[32], uint64_t delta) {
    unsigned carry = 0;
    for (int i = 0; i < 32; i++) {
        const unsigned add = i < 8 ? (unsigned)((delta >> (8 * i)) & 0xff) : 0u;
        if (!add && !carry && i >= 8) break;
        const unsigned s = sk[i] + add + carry;
        sk[i] = (uint8_t)s;
        carry = s >> 8;
    }
}

bool clamping_intact(const uint8_t sk[32]) {
    return (sk[0] & 7) == 0 && (sk[31] & 0xc0) == 0x40;
}

bool expanded_secret_at_offset(const uint8_t seed[32], uint64_t offset, uint8_t out[64]) {
    uint8_t e[64];
    expanded_secret_key(seed, e);
    add_to_scalar(e, offset);
    if (!clamping_intact(e)) return false;
    std::memcpy(out, e, 64);
    return true;
}

void block_seed(const uint8_t root[32], uint64_t index, uint8_t out[32]) {
    Sha512 h;
    static const char tag[] = "onion-gen block v1";
    h.update(tag, sizeof tag - 1);
    h.update(root, 32);
    uint8_t le[8];
    for (int i = 0; i < 8; i++) le[i] = (uint8_t)(index >> (8 * i));
    h.update(le, 8);
    uint8_t d[64];
    h.finish(d);
    std::memcpy(out, d, 32);
}

void checksum(const uint8_t pk[32], uint8_t out[2]) {
    uint8_t buf[48];
    std::memcpy(buf, ".onion checksum", 15);
    std::memcpy(buf + 15, pk, 32);
    buf[47] = 0x03;
    uint8_t d[32];
    sha3_256(buf, sizeof buf, d);
    out[0] = d[0];
    out[1] = d[1];
}

std::string address(const uint8_t pk[32]) {
    uint8_t b[35];
    std::memcpy(b, pk, 32);
    checksum(pk, b + 32);
    b[34] = 0x03;
    return base32_encode(b, 35);
}

void public_from_scalar(const uint8_t scalar[32], uint8_t pk[32]) { pt_encode(base_mult(scalar), pk); }

Pt start_point(const uint8_t seed[32]) {
    uint8_t sk[32];
    secret_scalar(seed, sk);
    return base_mult(sk);
}

HitCheck check_hit_scalar(const uint8_t scalar[32], uint64_t offset, const uint8_t packed[32], uint8_t pk[32]) {
    uint8_t sk[32];
    std::memcpy(sk, scalar, 32);
    add_to_scalar(sk, offset);
    if (!clamping_intact(sk)) return HitCheck::clamping;
    public_from_scalar(sk, pk);
    if (std::memcmp(pk, packed, 31) != 0 || (pk[31] & 0x7f) != (packed[31] & 0x7f)) return HitCheck::mismatch;
    return HitCheck::ok;
}

HitCheck check_hit(const uint8_t seed[32], uint64_t offset, const uint8_t packed[32], uint8_t pk[32],
                   uint8_t secret[64]) {
    uint8_t e[64];
    expanded_secret_key(seed, e);
    HitCheck c = check_hit_scalar(e, offset, packed, pk);
    if (c != HitCheck::ok) return c;
    add_to_scalar(e, offset);
    std::memcpy(secret, e, 64);
    return HitCheck::ok;
}

}  // namespace og
