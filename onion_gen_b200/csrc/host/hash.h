// SHA-512 (FIPS 180-4) and SHA3-256 (FIPS 202) for the host side of the
// engine: seed -> scalar derivation (src/key.rs:23-39), block seeds
// (src/run.rs:211-221) and the address checksum (src/key.rs:106-115).
#pragma once
#include <cstddef>
#include <cstdint>

namespace og {

class Sha512 {
public:
    Sha512();
    void update(const void* data, size_t len);
    void finish(uint8_t out[64]);

private:
    void block(const uint8_t* p);
    uint64_t h_[8];
    uint8_t buf_[128];
    size_t fill_ = 0;
    uint64_t total_ = 0;
};

void sha512(const void* data, size_t len, uint8_t out[64]);
void sha3_256(const void* data, size_t len, uint8_t out[32]);

}  // namespace og
