#include "ed25519.h"

#include <mutex>
#include <vector>

namespace og {

namespace {

// a^e for a 256-bit little-endian exponent (precompute only).
F51 f_pow(const F51& a, const uint8_t e[32]) {
    F51 r = f_one();
    for (int i = 255; i >= 0; i--) {
        r = f_sq(r);
        if ((e[i / 8] >> (i % 8)) & 1) r = f_mul(r, a);
    }
    return r;
}

// 2^k - c as a 256-bit little-endian exponent, for small c > 0.
void pow2_minus(uint8_t out[32], int k, unsigned c) {
    std::memset(out, 0, 32);
    // 2^k - 1 first: k one-bits.
    for (int i = 0; i < k; i++) out[i / 8] |= (uint8_t)(1u << (i % 8));
    // then subtract c - 1 from the low bytes (no borrow past them for small c).
    unsigned borrow = c - 1;
    for (int i = 0; i < 32 && borrow; i++) {
        unsigned cur = out[i], take = borrow & 0xff;
        borrow >>= 8;
        if (cur < take) {
            cur += 256;
            borrow += 1;
        }
        out[i] = (uint8_t)(cur - take);
    }
}

Pt make_basepoint() {
    // y = 4/5; x^2 = (y^2 - 1) / (d y^2 + 1); x taken even (RFC 8032 5.1).
    F51 four = f_zero(), five = f_zero();
    four.l[0] = 4;
    five.l[0] = 5;
    F51 y = f_mul(four, f_inv(five));
    F51 y2 = f_sq(y);
    F51 u = f_sub(y2, f_one());
    F51 v = f_add(f_mul(curve_d(), y2), f_one());
    F51 x2 = f_mul(u, f_inv(v));
    // candidate root x = x2^((p+3)/8), (p + 3) / 8 = 2^252 - 2
    uint8_t e[32];
    pow2_minus(e, 252, 2);
    F51 x = f_pow(x2, e);
    if (!f_equal(f_sq(x), x2)) {
        // sqrt(-1) = 2^((p-1)/4), (p - 1) / 4 = 2^253 - 5
        uint8_t q[32];
        pow2_minus(q, 253, 5);
        F51 two = f_zero();
        two.l[0] = 2;
        x = f_mul(x, f_pow(two, q));
    }
    if (f_is_odd(x)) x = f_sub(f_zero(), x);
    return Pt{x, y, f_one(), f_mul(x, y)};
}

struct BaseTable {
    Niels t[64][16];
};

const BaseTable& base_table() {
    static BaseTable* table = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        table = new BaseTable();
        Pt p = basepoint();
        for (int i = 0; i < 64; i++) {
            Pt acc = p;
            for (int j = 1; j < 16; j++) {
                table->t[i][j] = pt_niels(acc);
                acc = pt_add(acc, p);
            }
            for (int k = 0; k < 4; k++) p = pt_dbl(p);
        }
    });
    return *table;
}

}  // namespace

const Pt& basepoint() {
    static const Pt b = make_basepoint();
    return b;
}

Pt base_mult(const uint8_t scalar[32]) {
    const BaseTable& t = base_table();
    Pt acc = pt_identity();
    for (int i = 0; i < 64; i++) {
        const int nib = (scalar[i / 2] >> (4 * (i & 1))) & 15;
        if (nib) acc = pt_madd(acc, t.t[i][nib]);
    }
    return acc;
}

Pt base_mult_u64(uint64_t k) {
    uint8_t s[32] = {0};
    for (int i = 0; i < 8; i++) s[i] = (uint8_t)(k >> (8 * i));
    return base_mult(s);
}

Pt point_mult(const Pt& p, const uint8_t scalar[32]) {
    Pt acc = pt_identity();
    for (int i = 255; i >= 0; i--) {
        acc = pt_dbl(acc);
        if ((scalar[i / 8] >> (i % 8)) & 1) acc = pt_add(acc, p);
    }
    return acc;
}

}  // namespace og
