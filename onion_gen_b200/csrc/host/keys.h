// Keys, offsets and the address: the host side of the hit path.
//
// seed -> SHA-512 -> clamp -> scalar s (src/key.rs:23-51); the candidate at
// scalar offset o has secret s + o (src/key.rs:167-206); its address is
// base32(pk || SHA3-256(".onion checksum" || pk || 0x03)[0..2] || 0x03)
// (src/key.rs:106-132).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

#include "ed25519.h"

namespace og {

extern const char BASE32_ALPHABET[33];

int base32_value(char c);
std::string base32_encode(const uint8_t* bytes, size_t n);

void clamp_scalar(uint8_t sk[32]);
void secret_scalar(const uint8_t seed[32], uint8_t sk[32]);
void expanded_secret_key(const uint8_t seed[32], uint8_t out[64]);
void add_to_scalar(uint8_t sk[32], uint64_t delta);
bool clamping_intact(const uint8_t sk[32]);
// false when the offset carried into the clamped bits.
bool expanded_secret_at_offset(const uint8_t seed[32], uint64_t offset, uint8_t out[64]);
void block_seed(const uint8_t root[32], uint64_t index, uint8_t out[32]);

void checksum(const uint8_t pk[32], uint8_t out[2]);
std::string address(const uint8_t pk[32]);

// Public key (32 bytes, sign bit set) of a 32-byte scalar.
void public_from_scalar(const uint8_t scalar[32], uint8_t pk[32]);

// The start point of a seed: s * B.
Pt start_point(const uint8_t seed[32]);

// Re-derives the candidate at `offset` from the seed, independently of the
// device: the public key must equal the device's packed y in every bit but
// the sign (src/run.rs:1089-1104). On success fills the full public key
// (sign included) and the 64-byte expanded secret.
enum class HitCheck { ok = 0, clamping = 1, mismatch = 2 };
HitCheck check_hit(const uint8_t seed[32], uint64_t offset, const uint8_t packed[32], uint8_t pk[32],
                   uint8_t secret[64]);
// The same from a base scalar instead of a seed (secret half only).
HitCheck check_hit_scalar(const uint8_t scalar[32], uint64_t offset, const uint8_t packed[32], uint8_t pk[32]);

}  // namespace og
