// Host-side ed25519 for the engine: precompute (start points, strides,
// tables) and the independent re-derivation of every hit.
//
// Radix 2^51, five limbs, 128-bit products: a different representation from
// the device's eight 32-bit limbs, so that a hit re-derived here is checked by
// arithmetic that shares no code with the kernel that found it (the role
// curve25519-dalek plays for the reference, src/key.rs:76-94).
//
// Point formulas are the extended twisted-Edwards ones for a = -1
// (Hisil-Wong-Carter-Dawson 2008, as in RFC 8032 section 5.1.4).
#pragma once
#include <cstdint>
#include <cstring>

namespace og {

typedef unsigned __int128 u128;

struct F51 {
    uint64_t l[5];
};

static constexpr uint64_t M51 = (1ULL << 51) - 1;

inline F51 f_zero() { return F51{{0, 0, 0, 0, 0}}; }
inline F51 f_one() { return F51{{1, 0, 0, 0, 0}}; }

inline F51 f_carry(F51 a) {
    uint64_t c;
    for (int pass = 0; pass < 2; pass++) {
        c = a.l[0] >> 51; a.l[0] &= M51; a.l[1] += c;
        c = a.l[1] >> 51; a.l[1] &= M51; a.l[2] += c;
        c = a.l[2] >> 51; a.l[2] &= M51; a.l[3] += c;
        c = a.l[3] >> 51; a.l[3] &= M51; a.l[4] += c;
        c = a.l[4] >> 51; a.l[4] &= M51; a.l[0] += 19 * c;
    }
    return a;
}

inline F51 f_add(const F51& a, const F51& b) {
    F51 r;
    for (int i = 0; i < 5; i++) r.l[i] = a.l[i] + b.l[i];
    return f_carry(r);
}

// a - b + 4p keeps every limb positive for carried inputs.
inline F51 f_sub(const F51& a, const F51& b) {
    F51 r;
    r.l[0] = a.l[0] + 4 * (M51 - 18) - b.l[0];
    for (int i = 1; i < 5; i++) r.l[i] = a.l[i] + 4 * M51 - b.l[i];
    return f_carry(r);
}

inline F51 f_mul(const F51& a, const F51& b) {
    const uint64_t b1 = 19 * b.l[1], b2 = 19 * b.l[2], b3 = 19 * b.l[3], b4 = 19 * b.l[4];
    u128 t0 = (u128)a.l[0] * b.l[0] + (u128)a.l[1] * b4 + (u128)a.l[2] * b3 + (u128)a.l[3] * b2 + (u128)a.l[4] * b1;
    u128 t1 = (u128)a.l[0] * b.l[1] + (u128)a.l[1] * b.l[0] + (u128)a.l[2] * b4 + (u128)a.l[3] * b3 + (u128)a.l[4] * b2;
    u128 t2 = (u128)a.l[0] * b.l[2] + (u128)a.l[1] * b.l[1] + (u128)a.l[2] * b.l[0] + (u128)a.l[3] * b4 + (u128)a.l[4] * b3;
    u128 t3 = (u128)a.l[0] * b.l[3] + (u128)a.l[1] * b.l[2] + (u128)a.l[2] * b.l[1] + (u128)a.l[3] * b.l[0] + (u128)a.l[4] * b4;
    u128 t4 = (u128)a.l[0] * b.l[4] + (u128)a.l[1] * b.l[3] + (u128)a.l[2] * b.l[2] + (u128)a.l[3] * b.l[1] + (u128)a.l[4] * b.l[0];
    F51 r;
    t1 += (uint64_t)(t0 >> 51); r.l[0] = (uint64_t)t0 & M51;
    t2 += (uint64_t)(t1 >> 51); r.l[1] = (uint64_t)t1 & M51;
    t3 += (uint64_t)(t2 >> 51); r.l[2] = (uint64_t)t2 & M51;
    t4 += (uint64_t)(t3 >> 51); r.l[3] = (uint64_t)t3 & M51;
    uint64_t c = (uint64_t)(t4 >> 51); r.l[4] = (uint64_t)t4 & M51;
    r.l[0] += 19 * c;
    c = r.l[0] >> 51; r.l[0] &= M51; r.l[1] += c;
    return r;
}

inline F51 f_sq(const F51& a) { return f_mul(a, a); }

inline F51 f_sqn(F51 a, int n) {
    for (int i = 0; i < n; i++) a = f_sq(a);
    return a;
}

// a^(p-2) by the 2^255 - 21 addition chain.
inline F51 f_inv(const F51& z) {
    F51 z2 = f_sq(z);
    F51 z9 = f_mul(f_sqn(z2, 2), z);
    F51 z11 = f_mul(z9, z2);
    F51 e5 = f_mul(f_sq(z11), z9);
    F51 e10 = f_mul(f_sqn(e5, 5), e5);
    F51 e20 = f_mul(f_sqn(e10, 10), e10);
    F51 e40 = f_mul(f_sqn(e20, 20), e20);
    F51 e50 = f_mul(f_sqn(e40, 10), e10);
    F51 e100 = f_mul(f_sqn(e50, 50), e50);
    F51 e200 = f_mul(f_sqn(e100, 100), e100);
    F51 e250 = f_mul(f_sqn(e200, 50), e50);
    return f_mul(f_sqn(e250, 5), z11);
}

// 32 little-endian bytes; bit 255 is taken as part of the value (folded).
inline F51 f_from_bytes(const uint8_t b[32]) {
    uint64_t w[4];
    for (int k = 0; k < 4; k++) {
        uint64_t v = 0;
        for (int j = 7; j >= 0; j--) v = (v << 8) | b[8 * k + j];
        w[k] = v;
    }
    F51 r;
    r.l[0] = w[0] & M51;
    r.l[1] = ((w[0] >> 51) | (w[1] << 13)) & M51;
    r.l[2] = ((w[1] >> 38) | (w[2] << 26)) & M51;
    r.l[3] = ((w[2] >> 25) | (w[3] << 39)) & M51;
    r.l[4] = (w[3] >> 12) & M51;
    r.l[0] += 19 * (w[3] >> 63);
    return f_carry(r);
}

// Canonical encoding: fully reduce below p.
inline void f_to_bytes(F51 a, uint8_t out[32]) {
    a = f_carry(a);
    // q = 1 when a >= p: add 19 and look at bit 255.
    uint64_t q = (a.l[0] + 19) >> 51;
    q = (a.l[1] + q) >> 51;
    q = (a.l[2] + q) >> 51;
    q = (a.l[3] + q) >> 51;
    q = (a.l[4] + q) >> 51;
    a.l[0] += 19 * q;
    uint64_t c = a.l[0] >> 51; a.l[0] &= M51; a.l[1] += c;
    c = a.l[1] >> 51; a.l[1] &= M51; a.l[2] += c;
    c = a.l[2] >> 51; a.l[2] &= M51; a.l[3] += c;
    c = a.l[3] >> 51; a.l[3] &= M51; a.l[4] += c;
    a.l[4] &= M51;
    uint64_t w[4];
    w[0] = a.l[0] | (a.l[1] << 51);
    w[1] = (a.l[1] >> 13) | (a.l[2] << 38);
    w[2] = (a.l[2] >> 26) | (a.l[3] << 25);
    w[3] = (a.l[3] >> 39) | (a.l[4] << 12);
    for (int k = 0; k < 4; k++)
        for (int j = 0; j < 8; j++) out[8 * k + j] = (uint8_t)(w[k] >> (8 * j));
}

inline bool f_is_zero(const F51& a) {
    uint8_t b[32];
    f_to_bytes(a, b);
    uint8_t acc = 0;
    for (int i = 0; i < 32; i++) acc |= b[i];
    return acc == 0;
}

inline bool f_equal(const F51& a, const F51& b) { return f_is_zero(f_sub(a, b)); }

inline int f_is_odd(const F51& a) {
    uint8_t b[32];
    f_to_bytes(a, b);
    return b[0] & 1;
}

// The curve constant d = -121665/121666 and 2d.
inline const F51& curve_d() {
    static const F51 d = [] {
        F51 n = f_zero(), m = f_zero();
        n.l[0] = 121665;
        m.l[0] = 121666;
        return f_sub(f_zero(), f_mul(n, f_inv(m)));
    }();
    return d;
}

inline const F51& curve_2d() {
    static const F51 d2 = f_add(curve_d(), curve_d());
    return d2;
}

struct Pt {
    F51 X, Y, Z, T;
};

// Precomputed affine addend: (y + x, y - x, 2 d x y).
struct Niels {
    F51 ypx, ymx, xy2d;
};

inline Pt pt_identity() { return Pt{f_zero(), f_one(), f_one(), f_zero()}; }

// add-2008-hwcd-3 for a = -1.
inline Pt pt_add(const Pt& p, const Pt& q) {
    F51 A = f_mul(f_sub(p.Y, p.X), f_sub(q.Y, q.X));
    F51 B = f_mul(f_add(p.Y, p.X), f_add(q.Y, q.X));
    F51 C = f_mul(f_mul(p.T, curve_2d()), q.T);
    F51 D = f_mul(p.Z, q.Z);
    D = f_add(D, D);
    F51 E = f_sub(B, A), F = f_sub(D, C), G = f_add(D, C), H = f_add(B, A);
    return Pt{f_mul(E, F), f_mul(G, H), f_mul(F, G), f_mul(E, H)};
}

// mixed addition with an affine addend (Z = 1): madd-2008-hwcd-3.
inline Pt pt_madd(const Pt& p, const Niels& q) {
    F51 A = f_mul(f_sub(p.Y, p.X), q.ymx);
    F51 B = f_mul(f_add(p.Y, p.X), q.ypx);
    F51 C = f_mul(p.T, q.xy2d);
    F51 D = f_add(p.Z, p.Z);
    F51 E = f_sub(B, A), F = f_sub(D, C), G = f_add(D, C), H = f_add(B, A);
    return Pt{f_mul(E, F), f_mul(G, H), f_mul(F, G), f_mul(E, H)};
}

// dbl-2008-hwcd for a = -1.
inline Pt pt_dbl(const Pt& p) {
    F51 A = f_sq(p.X), B = f_sq(p.Y), C = f_sq(p.Z);
    C = f_add(C, C);
    F51 H = f_add(A, B);
    F51 E = f_sub(H, f_sq(f_add(p.X, p.Y)));
    F51 G = f_sub(A, B);
    F51 F = f_add(C, G);
    return Pt{f_mul(E, F), f_mul(G, H), f_mul(F, G), f_mul(E, H)};
}

inline Pt pt_neg(const Pt& p) { return Pt{f_sub(f_zero(), p.X), p.Y, p.Z, f_sub(f_zero(), p.T)}; }

inline void pt_affine(const Pt& p, F51& x, F51& y) {
    F51 zi = f_inv(p.Z);
    x = f_mul(p.X, zi);
    y = f_mul(p.Y, zi);
}

inline Niels pt_niels(const Pt& p) {
    F51 x, y;
    pt_affine(p, x, y);
    return Niels{f_add(y, x), f_sub(y, x), f_mul(f_mul(x, y), curve_2d())};
}

inline bool pt_equal(const Pt& a, const Pt& b) {
    return f_equal(f_mul(a.X, b.Z), f_mul(b.X, a.Z)) && f_equal(f_mul(a.Y, b.Z), f_mul(b.Y, a.Z));
}

// y with the sign of x in bit 255 (the ed25519 point encoding).
inline void pt_encode(const Pt& p, uint8_t out[32]) {
    F51 x, y;
    pt_affine(p, x, y);
    f_to_bytes(y, out);
    out[31] ^= (uint8_t)(f_is_odd(x) << 7);
}

// The base point: y = 4/5, x the even root.
const Pt& basepoint();

// scalar * B for a 256-bit little-endian scalar (not reduced), by 4-bit
// fixed windows over a table of j * 16^i * B built once per process.
Pt base_mult(const uint8_t scalar[32]);

// small * B.
Pt base_mult_u64(uint64_t k);

// scalar * P by double-and-add (slow; precompute only).
Pt point_mult(const Pt& p, const uint8_t scalar[32]);

}  // namespace og
