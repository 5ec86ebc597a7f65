/*
 * CPU oracle for the onion-gen key-search hot path — TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of onion-gen's CPU algorithms, used only by the test
 * suite, the smoke check and bench.py's CPU-baseline leg, as the checker or
 * as the timed CPU baseline. The product never links or calls it.
 *
 * Pinning: the field is checked against Python big-integer arithmetic, the
 * hashes against hashlib, and secret -> public -> address against the
 * reference's own stdlib-only Python verifier
 * (scripts/verify/verify-onion-address.py) through committed golden fixtures
 * under tests/golden/ (see make_golden.py there).
 *
 * Citations are file:line in the reference project.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <ctype.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef unsigned __int128 u128;

/* ========================================================================== */
/* Field: radix 2^64, four limbs, values below 2^256 folded with 2^256 = 38.  */
/* src/field.rs:13-266                                                         */
/* ========================================================================== */

typedef struct { uint64_t v[4]; } fe;

static const uint64_t MODULUS[4] = {
    0xffffffffffffffedULL, 0xffffffffffffffffULL,
    0xffffffffffffffffULL, 0x7fffffffffffffffULL};

static fe fe_zero(void) { fe r = {{0, 0, 0, 0}}; return r; }
static fe fe_one(void) { fe r = {{1, 0, 0, 0}}; return r; }

/* Fe::from_bytes (src/field.rs:35-43): top bit ignored. */
static fe fe_load(const uint8_t b[32]) {
    fe r;
    for (int k = 0; k < 4; k++) {
        uint64_t w = 0;
        for (int j = 7; j >= 0; j--) w = (w << 8) | b[8 * k + j];
        r.v[k] = w;
    }
    r.v[3] &= 0x7fffffffffffffffULL;
    return r;
}

/* the same, keeping bit 255 (for field tests on arbitrary 256-bit values). */
static fe fe_load_raw(const uint8_t b[32]) {
    fe r;
    for (int k = 0; k < 4; k++) {
        uint64_t w = 0;
        for (int j = 7; j >= 0; j--) w = (w << 8) | b[8 * k + j];
        r.v[k] = w;
    }
    return r;
}

/* Fe::to_bytes (src/field.rs:46-68): three conditional subtractions of p. */
static void fe_store(fe x, uint8_t out[32]) {
    for (int pass = 0; pass < 3; pass++) {
        uint64_t t[4], borrow = 0;
        for (int k = 0; k < 4; k++) {
            u128 d = (u128)x.v[k] - MODULUS[k] - borrow;
            t[k] = (uint64_t)d;
            borrow = (uint64_t)(d >> 64) & 1;
        }
        if (!borrow) memcpy(x.v, t, sizeof t);
    }
    for (int k = 0; k < 4; k++)
        for (int j = 0; j < 8; j++) out[8 * k + j] = (uint8_t)(x.v[k] >> (8 * j));
}

/* fold (src/field.rs:245-266): eight limbs -> four with 2^256 = 38, then two
 * unconditional passes for the carry that is left. */
static fe fe_fold(const uint64_t r[8]) {
    fe out;
    u128 c = 0;
    for (int k = 0; k < 4; k++) {
        u128 t = (u128)r[k] + (u128)38 * r[k + 4] + c;
        out.v[k] = (uint64_t)t;
        c = t >> 64;
    }
    uint64_t v = 38 * (uint64_t)c;
    for (int pass = 0; pass < 2; pass++) {
        for (int k = 0; k < 4; k++) {
            u128 s = (u128)out.v[k] + v;
            out.v[k] = (uint64_t)s;
            v = (uint64_t)(s >> 64);
        }
        v *= 38;
    }
    return out;
}

/* Fe::mul (src/field.rs:82-111): 4x4 schoolbook, row by row. */
static fe fe_mul(fe a, fe b) {
    uint64_t r[8] = {0};
    for (int i = 0; i < 4; i++) {
        uint64_t carry = 0;
        for (int j = 0; j < 4; j++) {
            u128 t = (u128)a.v[i] * b.v[j] + r[i + j] + carry;
            r[i + j] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        r[i + 4] = carry;
    }
    return fe_fold(r);
}

static fe fe_sq(fe a) { return fe_mul(a, a); }

/* add_small / sub_small (src/field.rs:270-307): two passes at most. */
static void add_small(uint64_t r[4], uint64_t v) {
    uint64_t carry = v;
    for (int pass = 0; pass < 2 && carry; pass++) {
        uint64_t c = carry;
        for (int k = 0; k < 4 && c; k++) {
            u128 s = (u128)r[k] + c;
            r[k] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        carry = 38 * c;
    }
}

static void sub_small(uint64_t r[4], uint64_t v) {
    uint64_t borrow = v;
    for (int pass = 0; pass < 2 && borrow; pass++) {
        uint64_t b = borrow;
        for (int k = 0; k < 4 && b; k++) {
            uint64_t d = r[k] - b;
            b = r[k] < b;
            r[k] = d;
        }
        borrow = 38 * b;
    }
}

/* Fe::add (src/field.rs:130-141). */
static fe fe_add(fe a, fe b) {
    fe r;
    uint64_t carry = 0;
    for (int k = 0; k < 4; k++) {
        u128 s = (u128)a.v[k] + b.v[k] + carry;
        r.v[k] = (uint64_t)s;
        carry = (uint64_t)(s >> 64);
    }
    add_small(r.v, 38 * carry);
    return r;
}

/* Fe::sub (src/field.rs:146-158). */
static fe fe_sub(fe a, fe b) {
    fe r;
    uint64_t borrow = 0;
    for (int k = 0; k < 4; k++) {
        u128 d = (u128)a.v[k] - b.v[k] - borrow;
        r.v[k] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    sub_small(r.v, 38 * borrow);
    return r;
}

static fe fe_sqn(fe a, int n) {
    for (int i = 0; i < n; i++) a = fe_sq(a);
    return a;
}

/* Fe::invert (src/field.rs:163-219): x^(p-2) by the ref10 addition chain,
 * 254 squarings and 11 multiplications. */
static fe fe_invert(fe z1) {
    fe z2 = fe_sq(z1);
    fe z8 = fe_sqn(z2, 2);
    fe z9 = fe_mul(z1, z8);
    fe z11 = fe_mul(z2, z9);
    fe z_5_0 = fe_mul(z9, fe_sq(z11));
    fe z_10_0 = fe_mul(fe_sqn(z_5_0, 5), z_5_0);
    fe z_20_0 = fe_mul(fe_sqn(z_10_0, 10), z_10_0);
    fe z_40_0 = fe_mul(fe_sqn(z_20_0, 20), z_20_0);
    fe z_50_0 = fe_mul(fe_sqn(z_40_0, 10), z_10_0);
    fe z_100_0 = fe_mul(fe_sqn(z_50_0, 50), z_50_0);
    fe z_200_0 = fe_mul(fe_sqn(z_100_0, 100), z_100_0);
    fe z_250_0 = fe_mul(fe_sqn(z_200_0, 50), z_50_0);
    return fe_mul(fe_sqn(z_250_0, 5), z11);
}

static int fe_is_negative(fe x) {
    uint8_t b[32];
    fe_store(x, b);
    return b[0] & 1;
}

static int fe_equal(fe a, fe b) {
    uint8_t x[32], y[32];
    fe_store(a, x);
    fe_store(b, y);
    return memcmp(x, y, 32) == 0;
}

void orc_fe_mul(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]) {
    fe_store(fe_mul(fe_load_raw(a), fe_load_raw(b)), out);
}
void orc_fe_sq(const uint8_t a[32], uint8_t out[32]) {
    fe_store(fe_sq(fe_load_raw(a)), out);
}
void orc_fe_add(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]) {
    fe_store(fe_add(fe_load_raw(a), fe_load_raw(b)), out);
}
void orc_fe_sub(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]) {
    fe_store(fe_sub(fe_load_raw(a), fe_load_raw(b)), out);
}
void orc_fe_invert(const uint8_t a[32], uint8_t out[32]) {
    fe_store(fe_invert(fe_load_raw(a)), out);
}
void orc_fe_canon(const uint8_t a[32], uint8_t out[32]) { fe_store(fe_load_raw(a), out); }

/* ========================================================================== */
/* Group: ed25519 in extended coordinates, src/curve.rs                        */
/* ========================================================================== */

typedef struct { fe x, y, z, t; } point;
typedef struct { fe ypx, ymx, z, t2d; } cached;
typedef struct { fe x, y, z, t; } p1p1;

static fe fe_hex(const char *h) {
    uint8_t b[32];
    for (int i = 0; i < 32; i++) {
        unsigned v;
        sscanf(h + 2 * i, "%2x", &v);
        b[i] = (uint8_t)v;
    }
    return fe_load(b);
}

/* Constants of src/curve.rs:28-39 (public ed25519 values, little-endian hex). */
#define HEX_BASE_X "1ad5258f602d56c9b2a7259560c72c695cdcd6fd31e2a4c0fe536ecdd3366921"
#define HEX_BASE_Y "5866666666666666666666666666666666666666666666666666666666666666"
#define HEX_8_YPX "8f3edd046659b7592c7088e27703b36c23c3d95e669c33b12fe5bc6160e71509"
#define HEX_8_YMX "d93492f3ed5da7e2f958b5e180763d96fb233c6eac41272cc3010e32a124903a"
#define HEX_8_T2D "1a91a2c9d9f5c1e7d7a7cc8b7871a3b8322ab60e19126463954ecc2e5c7c9026"
#define HEX_TWO_D "59f1b226949bd6eb56b183829a14e00030d1f3eef2808e19e7fcdf56dcd90624"

static point point_identity(void) {
    point p = {fe_zero(), fe_one(), fe_one(), fe_zero()};
    return p;
}

static point basepoint(void) {
    point p;
    p.x = fe_hex(HEX_BASE_X);
    p.y = fe_hex(HEX_BASE_Y);
    p.z = fe_one();
    p.t = fe_mul(p.x, p.y);
    return p;
}

static fe two_d(void) { return fe_hex(HEX_TWO_D); }

static cached eight_basepoint_cached(void) {
    cached c;
    c.ypx = fe_hex(HEX_8_YPX);
    c.ymx = fe_hex(HEX_8_YMX);
    c.z = fe_one();
    c.t2d = fe_hex(HEX_8_T2D);
    return c;
}

/* curve::add (src/curve.rs:130-144): p3 + cached -> p1p1, four multiplies. */
static p1p1 pt_add(const point *p, const cached *q) {
    fe a = fe_add(p->y, p->x);
    fe b = fe_sub(p->y, p->x);
    fe zz = fe_mul(a, q->ypx);
    fe yy = fe_mul(b, q->ymx);
    fe tt = fe_mul(q->t2d, p->t);
    fe t0 = fe_mul(p->z, q->z);
    t0 = fe_add(t0, t0);
    p1p1 r = {fe_sub(zz, yy), fe_add(zz, yy), fe_add(t0, tt), fe_sub(t0, tt)};
    return r;
}

/* curve::dbl (src/curve.rs:148-163). */
static p1p1 pt_dbl(const point *p) {
    fe xx = fe_sq(p->x);
    fe zz = fe_sq(p->y);
    fe tt = fe_sq(p->z);
    tt = fe_add(tt, tt);
    fe yy = fe_add(p->x, p->y);
    fe t0 = fe_sq(yy);
    fe y = fe_add(zz, xx);
    fe z = fe_sub(zz, xx);
    p1p1 r = {fe_sub(t0, y), y, z, fe_sub(tt, z)};
    return r;
}

/* curve::to_p3 (src/curve.rs:168-175). */
static point to_p3(const p1p1 *p) {
    point r = {fe_mul(p->x, p->t), fe_mul(p->y, p->z), fe_mul(p->z, p->t), fe_mul(p->x, p->y)};
    return r;
}

/* curve::to_cached (src/curve.rs:177-184). */
static cached to_cached(const point *p, fe td) {
    cached c = {fe_add(p->y, p->x), fe_sub(p->y, p->x), p->z, fe_mul(p->t, td)};
    return c;
}

static point add_p3(const point *p, const cached *q) {
    p1p1 s = pt_add(p, q);
    return to_p3(&s);
}

/* curve::scalar_base_mult (src/curve.rs:188-198): double-and-add from the top. */
static point scalar_mult(const uint8_t scalar[32], const point *base) {
    fe td = two_d();
    cached bc = to_cached(base, td);
    point acc = point_identity();
    for (int i = 255; i >= 0; i--) {
        p1p1 d = pt_dbl(&acc);
        acc = to_p3(&d);
        if ((scalar[i / 8] >> (i % 8)) & 1) acc = add_p3(&acc, &bc);
    }
    return acc;
}

static point scalar_base_mult(const uint8_t scalar[32]) {
    point b = basepoint();
    return scalar_mult(scalar, &b);
}

static void point_store(const point *p, uint8_t out[128]) {
    fe_store(p->x, out);
    fe_store(p->y, out + 32);
    fe_store(p->z, out + 64);
    fe_store(p->t, out + 96);
}

static point point_load(const uint8_t in[128]) {
    point p = {fe_load(in), fe_load(in + 32), fe_load(in + 64), fe_load(in + 96)};
    return p;
}

/* key::pack (src/key.rs:55-62). */
static void pack_point(const point *p, uint8_t out[32]) {
    fe zinv = fe_invert(p->z);
    fe y = fe_mul(p->y, zinv);
    fe x = fe_mul(p->x, zinv);
    fe_store(y, out);
    out[31] ^= (uint8_t)(fe_is_negative(x) << 7);
}

void orc_basepoint(uint8_t xyzt[128]) {
    point b = basepoint();
    point_store(&b, xyzt);
}

void orc_scalar_base_mult(const uint8_t scalar[32], uint8_t xyzt[128]) {
    point p = scalar_base_mult(scalar);
    point_store(&p, xyzt);
}

void orc_point_add(const uint8_t p[128], const uint8_t q[128], uint8_t out[128]) {
    point a = point_load(p), b = point_load(q);
    cached c = to_cached(&b, two_d());
    point r = add_p3(&a, &c);
    point_store(&r, out);
}

/* pairs.rs multiple_of_eight_g (src/pairs.rs:286-292). */
static point multiple_of_eight_g(uint64_t k) {
    uint8_t s[32] = {0};
    u128 prod = (u128)k * 8;
    for (int i = 0; i < 16; i++) s[i] = (uint8_t)(prod >> (8 * i));
    return scalar_base_mult(s);
}

void orc_multiple_of_eight_g(uint64_t k, uint8_t xyzt[128]) {
    point p = multiple_of_eight_g(k);
    point_store(&p, xyzt);
}

void orc_pack(const uint8_t xyzt[128], uint8_t out[32]) {
    point p = point_load(xyzt);
    pack_point(&p, out);
}

void orc_to_affine(const uint8_t xyzt[128], uint8_t x[32], uint8_t y[32]) {
    point p = point_load(xyzt);
    fe zinv = fe_invert(p.z);
    fe_store(fe_mul(p.x, zinv), x);
    fe_store(fe_mul(p.y, zinv), y);
}

static int is_identity(const point *p) {
    fe zinv = fe_invert(p->z);
    return fe_equal(fe_mul(p->x, zinv), fe_zero()) && fe_equal(fe_mul(p->y, zinv), fe_one());
}

/* curve.rs tests basepoint_has_expected_order (src/curve.rs:225). */
int orc_check_group_order(void) {
    static const uint8_t L[32] = {0xed, 0xd3, 0xf5, 0x5c, 0x1a, 0x63, 0x12, 0x58,
                                  0xd6, 0x9c, 0xf7, 0xa2, 0xde, 0xf9, 0xde, 0x14,
                                  0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0x10};
    point p = scalar_base_mult(L);
    return is_identity(&p);
}

/* curve.rs tests eight_basepoint_constant_matches_computed (src/curve.rs:231). */
int orc_check_eight_basepoint(void) {
    fe td = two_d();
    point b = basepoint();
    point e = b;
    for (int i = 0; i < 3; i++) {
        p1p1 d = pt_dbl(&e);
        e = to_p3(&d);
    }
    cached c = to_cached(&e, td);
    cached k = eight_basepoint_cached();
    fe zi = fe_invert(c.z), ki = fe_invert(k.z);
    return fe_equal(fe_mul(c.ypx, zi), fe_mul(k.ypx, ki)) &&
           fe_equal(fe_mul(c.ymx, zi), fe_mul(k.ymx, ki)) &&
           fe_equal(fe_mul(c.t2d, zi), fe_mul(k.t2d, ki));
}

/* ========================================================================== */
/* SHA-512, FIPS 180-4                                                          */
/* ========================================================================== */

/* First 64 bits of the fractional parts of the cube roots of the first 80
 * primes (FIPS 180-4 4.2.3). */
static const uint64_t SHA512_K[80] = {
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
/* Square roots of the first 8 primes (FIPS 180-4 5.3.5). */
static const uint64_t SHA512_H0[8] = {
    0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL, 0xa54ff53a5f1d36f1ULL,
    0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL, 0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL,
};

static uint64_t ror64(uint64_t x, int n) { return (x >> n) | (x << (64 - n)); }

static void sha512_block(uint64_t h[8], const uint8_t blk[128]) {
    uint64_t w[80];
    for (int i = 0; i < 16; i++) {
        uint64_t v = 0;
        for (int j = 0; j < 8; j++) v = (v << 8) | blk[8 * i + j];
        w[i] = v;
    }
    for (int i = 16; i < 80; i++) {
        uint64_t s0 = ror64(w[i - 15], 1) ^ ror64(w[i - 15], 8) ^ (w[i - 15] >> 7);
        uint64_t s1 = ror64(w[i - 2], 19) ^ ror64(w[i - 2], 61) ^ (w[i - 2] >> 6);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint64_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], k = h[7];
    for (int i = 0; i < 80; i++) {
        uint64_t S1 = ror64(e, 14) ^ ror64(e, 18) ^ ror64(e, 41);
        uint64_t ch = (e & f) ^ (~e & g);
        uint64_t t1 = k + S1 + ch + SHA512_K[i] + w[i];
        uint64_t S0 = ror64(a, 28) ^ ror64(a, 34) ^ ror64(a, 39);
        uint64_t maj = (a & b) ^ (a & c) ^ (b & c);
        uint64_t t2 = S0 + maj;
        k = g; g = f; f = e; e = d + t1;
        d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d;
    h[4] += e; h[5] += f; h[6] += g; h[7] += k;
}

void orc_sha512(const uint8_t *msg, size_t len, uint8_t out[64]) {
    uint64_t h[8];
    memcpy(h, SHA512_H0, sizeof h);
    size_t full = len / 128;
    for (size_t i = 0; i < full; i++) sha512_block(h, msg + 128 * i);
    uint8_t tail[256] = {0};
    size_t rem = len - 128 * full;
    memcpy(tail, msg + 128 * full, rem);
    tail[rem] = 0x80;
    size_t tl = (rem + 1 + 16 <= 128) ? 128 : 256;
    u128 bits = (u128)len * 8;
    for (int j = 0; j < 16; j++) tail[tl - 1 - j] = (uint8_t)(bits >> (8 * j));
    for (size_t off = 0; off < tl; off += 128) sha512_block(h, tail + off);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) out[8 * i + j] = (uint8_t)(h[i] >> (56 - 8 * j));
}

/* ========================================================================== */
/* SHA3-256, FIPS 202: Keccak-f[1600], rate 136, domain suffix 0x06            */
/* ========================================================================== */

static uint64_t rol64(uint64_t x, int n) { return n ? (x << n) | (x >> (64 - n)) : x; }

/* rc(t) of FIPS 202 3.2.5, the LFSR x^8 + x^6 + x^5 + x^4 + 1. */
static int keccak_rc_bit(int t) {
    if (t % 255 == 0) return 1;
    uint8_t r = 0x80;
    for (int i = 1; i <= t % 255; i++) {
        int r8 = r & 1;
        /* R = 0 || R, then R[0]^=R[8], R[4]^=R[8], R[5]^=R[8], R[6]^=R[8], truncate. */
        r >>= 1;
        if (r8) r ^= 0x80 | 0x08 | 0x04 | 0x02;
    }
    return (r >> 7) & 1;
}

static uint64_t keccak_rc[24];
static int keccak_rho[25];
static int keccak_ready;

static void keccak_init(void) {
    if (keccak_ready) return;
    for (int ir = 0; ir < 24; ir++) {
        uint64_t rc = 0;
        for (int j = 0; j <= 6; j++)
            if (keccak_rc_bit(j + 7 * ir)) rc |= 1ULL << ((1 << j) - 1);
        keccak_rc[ir] = rc;
    }
    /* rho offsets (FIPS 202 3.2.2). */
    keccak_rho[0] = 0;
    int x = 1, y = 0;
    for (int t = 0; t < 24; t++) {
        keccak_rho[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    keccak_ready = 1;
}

static void keccak_f(uint64_t a[25]) {
    for (int ir = 0; ir < 24; ir++) {
        uint64_t c[5], d[5], b[25];
        for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
        for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rol64(c[(x + 1) % 5], 1);
        for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
        /* rho and pi: B[y, 2x+3y] = rot(A[x, y], r[x, y]). */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++)
                b[y + 5 * ((2 * x + 3 * y) % 5)] = rol64(a[x + 5 * y], keccak_rho[x + 5 * y]);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= keccak_rc[ir];
    }
}

void orc_sha3_256(const uint8_t *msg, size_t len, uint8_t out[32]) {
    keccak_init();
    uint64_t a[25] = {0};
    const size_t rate = 136;
    uint8_t blk[136];
    size_t off = 0;
    for (;;) {
        size_t take = len - off < rate ? len - off : rate;
        memset(blk, 0, rate);
        memcpy(blk, msg + off, take);
        int last = take < rate;
        if (last) {
            blk[take] ^= 0x06;
            blk[rate - 1] ^= 0x80;
        }
        for (size_t i = 0; i < rate / 8; i++) {
            uint64_t v = 0;
            for (int j = 7; j >= 0; j--) v = (v << 8) | blk[8 * i + j];
            a[i] ^= v;
        }
        keccak_f(a);
        off += take;
        if (last) break;
    }
    for (int i = 0; i < 32; i++) out[i] = (uint8_t)(a[i / 8] >> (8 * (i % 8)));
}

/* ========================================================================== */
/* Keys, src/key.rs                                                             */
/* ========================================================================== */

static void clamp_bytes(uint8_t *sk) {
    sk[0] &= 248;
    sk[31] &= 63;
    sk[31] |= 64;
}

void orc_secret_scalar(const uint8_t seed[32], uint8_t sk[32]) {
    uint8_t d[64];
    orc_sha512(seed, 32, d);
    memcpy(sk, d, 32);
    clamp_bytes(sk);
}

void orc_expanded_secret_key(const uint8_t seed[32], uint8_t out[64]) {
    orc_sha512(seed, 32, out);
    clamp_bytes(out);
}

/* key::add_to_scalar (src/key.rs:185-195). */
void orc_add_to_scalar(uint8_t sk[32], uint64_t delta) {
    u128 carry = delta;
    for (int i = 0; i < 32 && carry; i++) {
        carry += sk[i];
        sk[i] = (uint8_t)carry;
        carry >>= 8;
    }
}

/* key::clamping_intact (src/key.rs:204-206). */
int orc_clamping_intact(const uint8_t sk[32]) {
    return (sk[0] & 248) == sk[0] && (((sk[31] & 63) | 64) == sk[31]);
}

/* key::expanded_secret_at_offset (src/key.rs:167-177). */
int orc_expanded_secret_at_offset(const uint8_t seed[32], uint64_t offset, uint8_t out[64]) {
    uint8_t e[64];
    orc_expanded_secret_key(seed, e);
    orc_add_to_scalar(e, offset);
    if (!orc_clamping_intact(e)) return 0;
    memcpy(out, e, 64);
    return 1;
}

void orc_public_key(const uint8_t seed[32], uint8_t out[32]) {
    uint8_t sk[32];
    orc_secret_scalar(seed, sk);
    point p = scalar_base_mult(sk);
    pack_point(&p, out);
}

/* key::checksum (src/key.rs:106-115). */
void orc_checksum(const uint8_t pk[32], uint8_t out[2]) {
    uint8_t buf[15 + 32 + 1], d[32];
    memcpy(buf, ".onion checksum", 15);
    memcpy(buf + 15, pk, 32);
    buf[47] = 0x03;
    orc_sha3_256(buf, sizeof buf, d);
    out[0] = d[0];
    out[1] = d[1];
}

/* ========================================================================== */
/* base32, src/base32.rs                                                        */
/* ========================================================================== */

static const char B32[] = "abcdefghijklmnopqrstuvwxyz234567";

static int symbol_value(char c) {
    if (c >= 'a' && c <= 'z') return c - 'a';
    if (c >= '2' && c <= '7') return c - '2' + 26;
    return -1;
}

size_t orc_base32_encode(const uint8_t *bytes, size_t n, char *out) {
    size_t o = 0;
    unsigned acc = 0, bits = 0;
    for (size_t i = 0; i < n; i++) {
        acc = ((acc << 8) | bytes[i]) & 0xffff;
        bits += 8;
        while (bits >= 5) {
            bits -= 5;
            out[o++] = B32[(acc >> bits) & 31];
        }
    }
    if (bits) out[o++] = B32[(acc << (5 - bits)) & 31];
    out[o] = 0;
    return o;
}

long orc_base32_decode_bits(const char *s, uint8_t *out, size_t cap, size_t *bits) {
    size_t o = 0, len = strlen(s);
    unsigned acc = 0, nb = 0;
    for (size_t i = 0; i < len; i++) {
        int v = symbol_value(s[i]);
        if (v < 0) return -(long)(i + 1);
        acc = ((acc << 5) | (unsigned)v) & 0xffff;
        nb += 5;
        if (nb >= 8) {
            nb -= 8;
            if (o < cap) out[o] = (uint8_t)(acc >> nb);
            o++;
        }
    }
    if (nb) {
        if (o < cap) out[o] = (uint8_t)(acc << (8 - nb));
        o++;
    }
    if (bits) *bits = len * 5;
    return (long)o;
}

void orc_address(const uint8_t pk[32], char out[57]) {
    uint8_t b[35];
    memcpy(b, pk, 32);
    orc_checksum(pk, b + 32);
    b[34] = 0x03;
    orc_base32_encode(b, 35, out);
}

/* run.rs block_seed (src/run.rs:211-221). */
void orc_block_seed(const uint8_t root[32], uint64_t index, uint8_t out[32]) {
    uint8_t buf[18 + 32 + 8], d[64];
    memcpy(buf, "onion-gen block v1", 18);
    memcpy(buf + 18, root, 32);
    for (int i = 0; i < 8; i++) buf[50 + i] = (uint8_t)(index >> (8 * i));
    orc_sha512(buf, sizeof buf, d);
    memcpy(out, d, 32);
}

/* ========================================================================== */
/* Chain engine, src/batch.rs:78-122                                            */
/* ========================================================================== */

typedef struct { fe x, y, z; } stored;

/* One BatchEngine::run: stores acc (without T), advances by 8G, then packs
 * the whole batch with one inversion (Montgomery). out gets the packed y
 * (sign clear); signs (nullable) gets the sign bit of x per element. */
static void chain_batch(point *acc, size_t n, stored *pts, fe *scratch,
                        uint8_t *out, uint8_t *signs) {
    cached step = eight_basepoint_cached();
    for (size_t i = 0; i < n; i++) {
        pts[i].x = acc->x;
        pts[i].y = acc->y;
        pts[i].z = acc->z;
        *acc = add_p3(acc, &step);
    }
    fe run = fe_one();
    for (size_t i = 0; i < n; i++) {
        scratch[i] = run;
        run = fe_mul(run, pts[i].z);
    }
    run = fe_invert(run);
    for (size_t i = n; i-- > 0;) {
        fe next = fe_mul(run, pts[i].z);
        fe zinv = fe_mul(run, scratch[i]);
        run = next;
        fe_store(fe_mul(pts[i].y, zinv), out + 32 * i);
        if (signs) signs[i] = (uint8_t)fe_is_negative(fe_mul(pts[i].x, zinv));
    }
}

static void chain_run(point *acc, size_t batch, size_t count, uint8_t *out, int with_sign) {
    stored *pts = malloc(batch * sizeof *pts);
    fe *scratch = malloc(batch * sizeof *scratch);
    uint8_t *buf = malloc(batch * 32);
    uint8_t *signs = malloc(batch);
    size_t done = 0;
    while (done < count) {
        chain_batch(acc, batch, pts, scratch, buf, with_sign ? signs : NULL);
        size_t take = count - done < batch ? count - done : batch;
        memcpy(out + 32 * done, buf, 32 * take);
        if (with_sign)
            for (size_t i = 0; i < take; i++) out[32 * (done + i) + 31] ^= (uint8_t)(signs[i] << 7);
        done += take;
    }
    free(pts);
    free(scratch);
    free(buf);
    free(signs);
}

void orc_chain_keys(const uint8_t start[128], size_t batch, size_t count, uint8_t *out,
                    uint8_t end[128]) {
    point acc = point_load(start);
    chain_run(&acc, batch, count, out, 0);
    if (end) point_store(&acc, end);
}

void orc_chain_keys_signed(const uint8_t start[128], size_t batch, size_t count, uint8_t *out) {
    point acc = point_load(start);
    chain_run(&acc, batch, count, out, 1);
}

typedef struct {
    point start;
    uint64_t first;
    size_t count;
    uint8_t *out;
} chain_job;

static void *chain_job_run(void *arg) {
    chain_job *j = arg;
    /* move to start + 8*first */
    point p = multiple_of_eight_g(j->first);
    cached c = to_cached(&p, two_d());
    point acc = add_p3(&j->start, &c);
    size_t batch = j->count < 4096 ? j->count : 4096;
    if (batch == 0) return NULL;
    chain_run(&acc, batch, j->count, j->out, 0);
    return NULL;
}

void orc_chain_keys_mt(const uint8_t start[128], uint64_t first, size_t count, uint8_t *out,
                       int threads) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    chain_job jobs[256];
    point s = point_load(start);
    size_t per = (count + threads - 1) / threads;
    int used = 0;
    for (int t = 0; t < threads; t++) {
        size_t lo = per * t;
        if (lo >= count) break;
        size_t n = count - lo < per ? count - lo : per;
        jobs[t].start = s;
        jobs[t].first = first + lo;
        jobs[t].count = n;
        jobs[t].out = out + 32 * lo;
        pthread_create(&th[t], NULL, chain_job_run, &jobs[t]);
        used++;
    }
    for (int t = 0; t < used; t++) pthread_join(th[t], NULL);
}

/* ========================================================================== */
/* Paired engine, src/pairs.rs:90-281                                           */
/* ========================================================================== */

typedef struct { fe x, y, xy; } affine;

typedef struct {
    size_t half, slots;
    affine *table;
    cached stride, to_first;
    fe *num, *den;
    uint64_t centre_delta;
    const uint64_t *probe; /* optional prefix bitmap tested per candidate */
    uint32_t probe_bits;
    uint64_t probe_hits;
} pair_engine;

/* pairs.rs to_affine_batch (src/pairs.rs:306-336). */
static void to_affine_batch(const point *pts, size_t n, affine *out) {
    fe *prefix = malloc(n * sizeof *prefix);
    fe run = fe_one();
    for (size_t i = 0; i < n; i++) {
        prefix[i] = run;
        run = fe_mul(run, pts[i].z);
    }
    fe inv = fe_invert(run);
    for (size_t i = n; i-- > 0;) {
        fe next = fe_mul(inv, pts[i].z);
        fe zinv = fe_mul(inv, prefix[i]);
        inv = next;
        out[i].x = fe_mul(pts[i].x, zinv);
        out[i].y = fe_mul(pts[i].y, zinv);
        out[i].xy = fe_mul(out[i].x, out[i].y);
    }
    free(prefix);
}

/* PairEngine::new (src/pairs.rs:90-137). */
static void pair_new(pair_engine *e, size_t half) {
    e->half = half;
    e->slots = 2 * half + 1;
    cached step = eight_basepoint_cached();
    point *pts = malloc(half * sizeof *pts);
    point id = point_identity();
    point p = add_p3(&id, &step);
    for (size_t i = 0; i < half; i++) {
        pts[i] = p;
        p = add_p3(&p, &step);
    }
    e->table = malloc(half * sizeof *e->table);
    to_affine_batch(pts, half, e->table);
    free(pts);
    point s = multiple_of_eight_g(2 * half + 1);
    point f = multiple_of_eight_g(half + 1);
    e->stride = to_cached(&s, two_d());
    e->to_first = to_cached(&f, two_d());
    e->num = malloc(e->slots * sizeof(fe));
    e->den = malloc(e->slots * sizeof(fe));
    e->centre_delta = 0;
    e->probe = NULL;
    e->probe_bits = 0;
    e->probe_hits = 0;
}

static void pair_free(pair_engine *e) {
    free(e->table);
    free(e->num);
    free(e->den);
}

/* PairEngine::begin (src/pairs.rs:146-150). */
static void pair_begin(pair_engine *e, point *acc) {
    *acc = add_p3(acc, &e->to_first);
    e->centre_delta = 8 * (e->half + 1);
}

/* PairEngine::delta (src/pairs.rs:234-247), for the round just run. */
static uint64_t pair_delta(const pair_engine *e, size_t index) {
    uint64_t centre = e->centre_delta - 8 * (2 * e->half + 1);
    if (index == 2 * e->half) return centre;
    uint64_t m = 8 * (index / 2 + 1);
    return (index % 2 == 0) ? centre + m : centre - m;
}

/* PairEngine::run_inner with no probe (src/pairs.rs:174-224): every
 * candidate's y, written by index (keys nullable). */
static void pair_run(pair_engine *e, point *acc, uint8_t *keys) {
    size_t half = e->half, n = e->slots;
    fe zinv = fe_invert(acc->z);
    affine pa;
    pa.x = fe_mul(acc->x, zinv);
    pa.y = fe_mul(acc->y, zinv);
    pa.xy = fe_mul(pa.x, pa.y);
    fe run = fe_one();
    for (size_t j = 0; j < half; j++) {
        const affine *q = &e->table[j];
        fe x1y2 = fe_mul(pa.x, q->y);
        fe y1x2 = fe_mul(pa.y, q->x);
        fe d0 = fe_sub(x1y2, y1x2);
        e->num[2 * j] = fe_mul(fe_sub(pa.xy, q->xy), run);
        e->den[2 * j] = d0;
        run = fe_mul(run, d0);
        fe d1 = fe_add(x1y2, y1x2);
        e->num[2 * j + 1] = fe_mul(fe_add(pa.xy, q->xy), run);
        e->den[2 * j + 1] = d1;
        run = fe_mul(run, d1);
    }
    e->num[n - 1] = fe_mul(pa.y, run);
    e->den[n - 1] = fe_one();
    fe inv = fe_invert(run);
    for (size_t i = n; i-- > 0;) {
        fe v = fe_mul(inv, e->num[i]);
        inv = fe_mul(inv, e->den[i]);
        if (keys) {
            fe_store(v, keys + 32 * i);
        } else if (e->probe) {
            /* LimbProbe::may_match (src/filter.rs:2615-2633): the first limb
             * and the two values canonicalising can turn it into. */
            uint64_t l0 = v.v[0];
            for (int k = 0; k < 3; k++, l0 += 19) {
                uint64_t head = __builtin_bswap64(l0);
                size_t slot = (size_t)(head >> (64 - e->probe_bits));
                if ((e->probe[slot >> 6] >> (slot & 63)) & 1) {
                    uint8_t b[32];
                    fe_store(v, b);
                    e->probe_hits++;
                    break;
                }
            }
        }
    }
    *acc = add_p3(acc, &e->stride);
    e->centre_delta += 8 * (2 * half + 1);
}

void orc_pair_keys(const uint8_t start[128], size_t half, size_t rounds, uint8_t *keys,
                   uint64_t *deltas) {
    pair_engine e;
    pair_new(&e, half);
    point acc = point_load(start);
    pair_begin(&e, &acc);
    for (size_t r = 0; r < rounds; r++) {
        uint8_t *k = keys ? keys + 32 * e.slots * r : NULL;
        pair_run(&e, &acc, k);
        if (deltas)
            for (size_t i = 0; i < e.slots; i++) deltas[e.slots * r + i] = pair_delta(&e, i);
    }
    pair_free(&e);
}

/* ---- CPU throughput, the src/estimate.rs:86-117 method ------------------- */

typedef struct {
    int which; /* 0 pair, 1 chain */
    size_t size;
    double seconds;
    uint64_t seed;
    uint64_t examined;
    double elapsed;
    /* one search (orc_pair_rate_search): its seed, its index, the thread's
     * place in it */
    const uint8_t *search_seed;
    const uint64_t *bitmap;
    uint32_t bits;
    int index;
} rate_job;

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void *rate_run(void *arg) {
    rate_job *j = arg;
    uint8_t seed[32] = {0};
    for (int i = 0; i < 8; i++) seed[i] = (uint8_t)(j->seed >> (8 * i));
    uint8_t sk[32];
    orc_secret_scalar(j->search_seed ? j->search_seed : seed, sk);
    point acc = scalar_base_mult(sk);
    if (j->search_seed && j->index > 0) {
        /* thread t starts 2^40 t candidates into the search */
        const point off = multiple_of_eight_g((uint64_t)j->index << 40);
        const cached c = to_cached(&off, two_d());
        acc = add_p3(&acc, &c);
    }
    if (j->which == 0) {
        pair_engine e;
        pair_new(&e, j->size);
        /* a 16-bit index with one slot set, as a six-symbol prefix makes,
         * unless the search's own index is given */
        uint64_t *bm = NULL;
        if (j->bitmap) {
            e.probe = j->bitmap;
            e.probe_bits = j->bits;
        } else {
            bm = calloc(1024, sizeof *bm);
            bm[j->seed % 1024] = 1;
            e.probe = bm;
            e.probe_bits = 16;
        }
        pair_begin(&e, &acc);
        pair_run(&e, &acc, NULL); /* untimed round */
        double t0 = now_s();
        uint64_t n = 0;
        do {
            pair_run(&e, &acc, NULL);
            n += e.slots;
        } while (now_s() - t0 < j->seconds);
        j->elapsed = now_s() - t0;
        j->examined = n;
        pair_free(&e);
        free(bm);
    } else {
        size_t b = j->size;
        stored *pts = malloc(b * sizeof *pts);
        fe *scratch = malloc(b * sizeof *scratch);
        uint8_t *buf = malloc(b * 32);
        chain_batch(&acc, b, pts, scratch, buf, NULL);
        double t0 = now_s();
        uint64_t n = 0;
        do {
            chain_batch(&acc, b, pts, scratch, buf, NULL);
            n += b;
        } while (now_s() - t0 < j->seconds);
        j->elapsed = now_s() - t0;
        j->examined = n;
        free(pts);
        free(scratch);
        free(buf);
    }
    return NULL;
}

static double rate_common(int which, int threads, double seconds, size_t size, const uint8_t *search_seed,
                          const uint64_t *bitmap, uint32_t bits, uint64_t *examined) {
    if (threads < 1) threads = 1;
    if (threads > 512) threads = 512;
    pthread_t *th = calloc(threads, sizeof *th);
    rate_job *jobs = calloc(threads, sizeof *jobs);
    for (int t = 0; t < threads; t++) {
        jobs[t].which = which;
        jobs[t].size = size;
        jobs[t].seconds = seconds;
        jobs[t].seed = 0x6f6e696f6e000000ULL + (uint64_t)t;
        jobs[t].search_seed = search_seed;
        jobs[t].bitmap = bitmap;
        jobs[t].bits = bits;
        jobs[t].index = t;
        pthread_create(&th[t], NULL, rate_run, &jobs[t]);
    }
    double rate = 0;
    uint64_t total = 0;
    for (int t = 0; t < threads; t++) {
        pthread_join(th[t], NULL);
        total += jobs[t].examined;
        if (jobs[t].elapsed > 0) rate += jobs[t].examined / jobs[t].elapsed;
    }
    free(th);
    free(jobs);
    if (examined) *examined = total;
    return rate;
}

double orc_pair_rate(int threads, double seconds, size_t half, uint64_t *examined) {
    return rate_common(0, threads, seconds, half, NULL, NULL, 0, examined);
}

double orc_pair_rate_search(int threads, double seconds, size_t half, const uint8_t seed[32], const uint64_t *bitmap,
                            uint32_t bits, uint64_t *examined) {
    if (!seed || !bitmap || bits < 1 || bits > 32) {
        if (examined) *examined = 0;
        return 0;
    }
    return rate_common(0, threads, seconds, half, seed, bitmap, bits, examined);
}

double orc_chain_rate(int threads, double seconds, size_t batch, uint64_t *examined) {
    return rate_common(1, threads, seconds, batch, NULL, NULL, 0, examined);
}

/* ========================================================================== */
/* Filters: literal prefixes, src/filter.rs                                     */
/* ========================================================================== */

#define KEY_ONLY_SYMBOLS 49 /* src/filter.rs:134 */
#define ADDRESS_LEN 56      /* src/key.rs:19 */

typedef struct {
    char canonical[ADDRESS_LEN * 34 + 1];
    size_t len;
    uint8_t bytes[32];
    size_t nbytes;
    uint8_t mask;
    int pattern;           /* a prefix with `?` or `[...]`: matched by sets */
    uint32_t sets[ADDRESS_LEN];
} ofilter;

static int parse_symbol_body(const char *s, size_t a, size_t b, uint32_t *sets, size_t *n, char *err, size_t errlen);
static size_t render_symbol_sets(const uint32_t *sets, size_t n, char *out);
static unsigned orc_symbol_at(const uint8_t *b, size_t len, size_t pos);

struct orc_fset {
    ofilter *f;
    size_t n;
    uint32_t bits;
    uint64_t *words;
    size_t nwords;
};

/* Pattern::parse + Filter::parse (src/filter.rs:298-352, 649-685) for the
 * literal-prefix form: trim, optional "prefix:" or leading '^', lowercase,
 * every symbol in the alphabet. Other forms are outside this oracle. */
static int parse_literal(const char *raw, size_t rawlen, ofilter *out, char *err, size_t errlen) {
    while (rawlen && (*raw == ' ' || *raw == '\t' || *raw == '\r')) raw++, rawlen--;
    while (rawlen && (raw[rawlen - 1] == ' ' || raw[rawlen - 1] == '\t' || raw[rawlen - 1] == '\r'))
        rawlen--;
    char buf[256];
    if (rawlen >= sizeof buf) {
        snprintf(err, errlen, "filter too long");
        return -1;
    }
    memcpy(buf, raw, rawlen);
    buf[rawlen] = 0;
    char *body = buf;
    char *colon = strchr(buf, ':');
    if (colon) {
        *colon = 0;
        char *name = buf;
        while (*name == ' ') name++;
        for (char *p = name; *p; p++)
            if (*p >= 'A' && *p <= 'Z') *p = (char)(*p - 'A' + 'a');
        size_t nl = strlen(name);
        while (nl && name[nl - 1] == ' ') name[--nl] = 0;
        if (strcmp(name, "prefix") != 0) {
            snprintf(err, errlen, "only literal prefixes are supported, got form %s", name);
            return -1;
        }
        body = colon + 1;
        while (*body == ' ') body++;
        size_t bl = strlen(body);
        while (bl && body[bl - 1] == ' ') body[--bl] = 0;
    } else {
        while (*body == '^') body++;
    }
    size_t n = strlen(body);
    if (n == 0) {
        snprintf(err, errlen, "the filter is empty");
        return -1;
    }
    out->pattern = strpbrk(body, "?[]") != NULL;
    if (out->pattern) {
        /* Pattern::parse with wildcards or classes (src/filter.rs:298-350,
         * parse_symbols :495-560), anchored at the start */
        size_t m = 0;
        if (parse_symbol_body(body, 0, n, out->sets, &m, err, errlen) != 0) return -1;
        int fixed = 0;
        for (size_t i = 0; i < m; i++) fixed |= out->sets[i] != 0xffffffffu;
        if (!fixed) {
            snprintf(err, errlen, "nothing fixed");
            return -1;
        }
        out->len = m;
        render_symbol_sets(out->sets, m, out->canonical);
        out->nbytes = 0;
        return 0;
    }
    if (n > ADDRESS_LEN) {
        snprintf(err, errlen, "filter of %zu symbols is longer than an address", n);
        return -1;
    }
    for (size_t i = 0; i < n; i++) {
        char c = body[i];
        if (c >= 'A' && c <= 'Z') c = (char)(c - 'A' + 'a');
        if (symbol_value(c) < 0) {
            snprintf(err, errlen, "invalid character '%c' at position %zu", body[i], i);
            return -1;
        }
        out->canonical[i] = c;
    }
    out->canonical[n] = 0;
    out->len = n;
    char head[KEY_ONLY_SYMBOLS + 1];
    size_t hn = n < KEY_ONLY_SYMBOLS ? n : KEY_ONLY_SYMBOLS;
    memcpy(head, out->canonical, hn);
    head[hn] = 0;
    uint8_t dec[40];
    size_t bits;
    orc_base32_decode_bits(head, dec, sizeof dec, &bits);
    size_t significant = (bits + 7) / 8;
    unsigned rem = bits % 8;
    out->mask = rem == 0 ? 0xff : (uint8_t)(0xff << (8 - rem));
    memcpy(out->bytes, dec, significant);
    out->nbytes = significant;
    out->bytes[significant - 1] &= out->mask;
    return 0;
}

static int cmp_canonical(const void *a, const void *b) {
    return strcmp(((const ofilter *)a)->canonical, ((const ofilter *)b)->canonical);
}

/* BitmapIndex::slot with offset 0 (src/filter.rs:2538-2549). */
static size_t bitmap_slot(uint32_t bits, const uint8_t packed[32]) {
    uint64_t w = 0;
    for (int i = 0; i < 8; i++) w = (w << 8) | packed[i];
    return (size_t)(w >> (64 - bits));
}

static double words_occupancy(const uint64_t *w, size_t nw, uint32_t bits) {
    uint64_t set = 0;
    for (size_t i = 0; i < nw; i++) set += (uint64_t)__builtin_popcountll(w[i]);
    return (double)set / (double)(1ULL << bits);
}

/* BitmapIndex::build + insert (src/filter.rs:2334-2351, 2552-2578). Returns
 * NULL when the map would be more than a quarter full. */
static uint64_t *bitmap_build(const ofilter *f, size_t n, uint32_t bits, size_t *nwords) {
    if (n == 0 || bits < 8 || bits > 32) return NULL;
    size_t nw = (size_t)(((1ULL << bits) + 63) / 64);
    uint64_t *w = calloc(nw, sizeof *w);
    for (size_t i = 0; i < n; i++) {
        if (f[i].pattern) {
            /* pattern_slots (src/filter.rs:2480-2530): every slot the sets
             * allow over the window's first bits / 5 symbols and the top
             * bits % 5 bits of the next; more than 4096 cannot be indexed */
            uint32_t full = bits / 5, rem = bits % 5;
            size_t nv = 1;
            uint32_t *vals = malloc(sizeof *vals);
            vals[0] = 0;
            for (uint32_t k = 0; k <= full; k++) {
                if (k == full && rem == 0) break;
                uint32_t set = k < f[i].len ? f[i].sets[k] : 0xffffffffu;
                uint32_t parts = 0;
                for (unsigned v = 0; v < 32; v++)
                    if ((set >> v) & 1) parts |= 1u << (k < full ? v : (v >> (5 - rem)));
                size_t np = (size_t)__builtin_popcount(parts);
                if (nv * np > 4096) {
                    free(vals);
                    free(w);
                    return NULL;
                }
                uint32_t shift = k < full ? bits - 5 * (k + 1) : 0;
                uint32_t *next = malloc(nv * np * sizeof *next);
                size_t q = 0;
                for (size_t a = 0; a < nv; a++)
                    for (unsigned part = 0; part < 32; part++)
                        if ((parts >> part) & 1) next[q++] = vals[a] | (part << shift);
                free(vals);
                vals = next;
                nv = q;
            }
            for (size_t a = 0; a < nv; a++) w[vals[a] >> 6] |= 1ULL << (vals[a] & 63);
            free(vals);
            continue;
        }
        size_t sym = f[i].len < KEY_ONLY_SYMBOLS ? f[i].len : KEY_ONLY_SYMBOLS;
        uint32_t pbits = (uint32_t)(sym * 5);
        uint8_t probe[32] = {0};
        memcpy(probe, f[i].bytes, f[i].nbytes);
        size_t first = bitmap_slot(bits, probe);
        size_t run = pbits >= bits ? 1 : ((size_t)1 << (bits - pbits));
        for (size_t s = first; s < first + run; s++) w[s >> 6] |= 1ULL << (s & 63);
    }
    if (words_occupancy(w, nw, bits) > 0.25) {
        free(w);
        return NULL;
    }
    *nwords = nw;
    return w;
}

orc_fset *orc_fset_new(const char *text, uint32_t bits, char *err, size_t errlen) {
    size_t cap = 16, n = 0;
    ofilter *f = malloc(cap * sizeof *f);
    const char *p = text;
    while (*p) {
        const char *e = strchr(p, '\n');
        size_t len = e ? (size_t)(e - p) : strlen(p);
        int blank = 1;
        for (size_t i = 0; i < len; i++)
            if (p[i] != ' ' && p[i] != '\t' && p[i] != '\r') blank = 0;
        if (!blank) {
            if (n == cap) f = realloc(f, (cap *= 2) * sizeof *f);
            if (parse_literal(p, len, &f[n], err, errlen) != 0) {
                free(f);
                return NULL;
            }
            n++;
        }
        if (!e) break;
        p = e + 1;
    }
    /* FilterSet::new (src/filter.rs:1326-1339): sort, drop absorbed. */
    qsort(f, n, sizeof *f, cmp_canonical);
    size_t kept = 0;
    long last_literal = -1;
    for (size_t i = 0; i < n; i++) {
        if (f[i].pattern) {
            /* patterns: exact duplicates only */
            int dup = 0;
            for (size_t j = 0; j < kept && !dup; j++)
                dup = f[j].pattern && strcmp(f[j].canonical, f[i].canonical) == 0;
            if (!dup) f[kept++] = f[i];
            continue;
        }
        if (last_literal >= 0 &&
            strncmp(f[i].canonical, f[last_literal].canonical, f[last_literal].len) == 0)
            continue;
        last_literal = (long)kept;
        f[kept++] = f[i];
    }
    orc_fset *s = calloc(1, sizeof *s);
    s->f = f;
    s->n = kept;
    if (bits == 0) {
        /* narrowest_acceptable (src/filter.rs:2279-2295), target 0.01. */
        uint64_t *widest = NULL;
        size_t widest_n = 0;
        uint32_t widest_bits = 0;
        for (uint32_t b = 16; b <= 24; b++) {
            size_t nw;
            uint64_t *w = bitmap_build(f, kept, b, &nw);
            if (!w) continue;
            if (words_occupancy(w, nw, b) <= 0.01) {
                free(widest);
                widest = w;
                widest_n = nw;
                widest_bits = b;
                break;
            }
            free(widest);
            widest = w;
            widest_n = nw;
            widest_bits = b;
        }
        s->words = widest;
        s->nwords = widest_n;
        s->bits = widest_bits;
    } else {
        s->words = bitmap_build(f, kept, bits, &s->nwords);
        s->bits = bits;
    }
    if (!s->words) {
        snprintf(err, errlen, "no prefix index could be built");
        free(f);
        free(s);
        return NULL;
    }
    return s;
}

void orc_fset_free(orc_fset *s) {
    if (!s) return;
    free(s->f);
    free(s->words);
    free(s);
}

size_t orc_fset_count(const orc_fset *s) { return s->n; }
void orc_fset_canonical(const orc_fset *s, size_t i, char *out, size_t cap) {
    snprintf(out, cap, "%s", s->f[i].canonical);
}
uint32_t orc_fset_bits(const orc_fset *s) { return s->bits; }
size_t orc_fset_nwords(const orc_fset *s) { return s->nwords; }
const uint64_t *orc_fset_words(const orc_fset *s) { return s->words; }
double orc_fset_occupancy(const orc_fset *s) { return words_occupancy(s->words, s->nwords, s->bits); }

/* BitmapIndex::may_match (src/filter.rs:2581-2585). */
int orc_fset_may_match(const orc_fset *s, const uint8_t packed[32]) {
    size_t slot = bitmap_slot(s->bits, packed);
    return (int)((s->words[slot >> 6] >> (slot & 63)) & 1);
}

/* FilterSet::match_key for literal prefixes (src/filter.rs:2098-2213,
 * 819-834): bitmap, then a masked byte compare. A scan stands in for the
 * length buckets; it returns the same filter because the kept set holds no
 * filter absorbed by another, so at most one can match. */
long orc_fset_match(const orc_fset *s, const uint8_t packed[32]) {
    if (!orc_fset_may_match(s, packed)) return -1;
    for (size_t i = 0; i < s->n; i++) {
        const ofilter *f = &s->f[i];
        if (f->pattern) continue;
        size_t last = f->nbytes - 1;
        if (memcmp(packed, f->bytes, last) == 0 && (packed[last] & f->mask) == f->bytes[last])
            return (long)i;
    }
    /* patterns, in order, on the key-only symbols (src/filter.rs:760-770) */
    for (size_t i = 0; i < s->n; i++) {
        const ofilter *f = &s->f[i];
        if (!f->pattern) continue;
        size_t k, m = f->len < KEY_ONLY_SYMBOLS ? f->len : KEY_ONLY_SYMBOLS;
        for (k = 0; k < m; k++)
            if (!((f->sets[k] >> orc_symbol_at(packed, 32, k)) & 1)) break;
        if (k == m) return (long)i;
    }
    return -1;
}

/* ========================================================================== */
/* Reference device bookkeeping                                                 */
/* ========================================================================== */

/* src/gpu/cuda.rs:332-354. */
uint64_t orc_cuda_offset(uint64_t tid, uint64_t slot, uint64_t launch, uint32_t threads,
                         uint32_t half) {
    uint64_t slots = 2 * (uint64_t)half + 1;
    uint64_t window = tid + launch * threads;
    uint64_t centre = (window * slots + half + 1) * 8;
    if (slot == slots - 1) return centre;
    uint64_t stepped = (slot / 2 + 1) * 8;
    return slot % 2 == 0 ? centre + stepped : centre - stepped;
}

/* src/gpu/mod.rs:306-312. */
uint32_t orc_hit_room(uint64_t batch, uint32_t bits) {
    uint64_t expected = batch >> (bits < 63 ? bits : 63);
    uint64_t v = expected > (UINT64_MAX - 1024) / 4 ? UINT64_MAX : expected * 4 + 1024;
    if (v < 4096) v = 4096;
    if (v > (1u << 18)) v = 1u << 18;
    return (uint32_t)v;
}

/* ========================================================================== */
/* Suffix filters, src/filter.rs (the `suffix:` form)                          */
/* ========================================================================== */

#define ORC_ALL 0xffffffffu

typedef struct {
    uint32_t sets[56];
    size_t len;
    char text[64 * 34];
} osuffix;

struct orc_sset {
    osuffix *p;
    size_t n;
    uint32_t bits;
    uint64_t *words;
    size_t nwords;
};

/* either_sign (src/filter.rs:158-164): symbol 49 holds the sign bit at
 * weight 2, so each value pairs with the one two away in its group of four. */
static uint32_t orc_either_sign(uint32_t set) {
    uint32_t out = set;
    for (unsigned v = 0; v < 32; v++)
        if ((set >> v) & 1) out |= 1u << (v ^ 2);
    return out;
}

/* symbol_at (src/filter.rs:259-267) over a buffer of `len` bytes. */
static unsigned orc_symbol_at(const uint8_t *b, size_t len, size_t pos) {
    unsigned v = 0;
    for (unsigned k = 0; k < 5; k++) {
        size_t bit = pos * 5 + k;
        unsigned x = bit / 8 < len ? (b[bit / 8] >> (7 - bit % 8)) & 1 : 0;
        v = (v << 1) | x;
    }
    return v;
}

/* Pattern::parse for a suffix body (src/filter.rs:298-350, parse_symbols
 * :495-560, check_reachable_tail :566-600). */
/* parse_symbols (src/filter.rs:495-560): one symbol set per position,
 * from s[a..b): a symbol, `?`, or a `[...]` class with `x-y` ranges. */
static int parse_symbol_body(const char *s, size_t a, size_t b, uint32_t *sets, size_t *count, char *err,
                             size_t errlen) {
    size_t n = 0;
    for (size_t i = a; i < b;) {
        uint32_t set = 0;
        if (s[i] == '?') {
            set = ORC_ALL;
            i++;
        } else if (s[i] == '[') {
            size_t e = i + 1;
            while (e < b && s[e] != ']') e++;
            if (e == b) { snprintf(err, errlen, "unbalanced class"); return -1; }
            for (size_t j = i + 1; j < e;) {
                int f = symbol_value((char)tolower((unsigned char)s[j]));
                if (f < 0) { snprintf(err, errlen, "bad symbol"); return -1; }
                if (j + 2 < e && s[j + 1] == '-') {
                    int l = symbol_value((char)tolower((unsigned char)s[j + 2]));
                    if (l < 0) { snprintf(err, errlen, "bad symbol"); return -1; }
                    if (l < f) { snprintf(err, errlen, "empty range"); return -1; }
                    for (int v = f; v <= l; v++) set |= 1u << v;
                    j += 3;
                } else {
                    set |= 1u << f;
                    j++;
                }
            }
            if (!set) { snprintf(err, errlen, "empty class"); return -1; }
            i = e + 1;
        } else {
            int v = symbol_value((char)tolower((unsigned char)s[i]));
            if (v < 0) { snprintf(err, errlen, "bad symbol"); return -1; }
            set = 1u << v;
            i++;
        }
        if (n == 56) { snprintf(err, errlen, "too long"); return -1; }
        sets[n++] = set;
    }
    *count = n;
    return 0;
}

static size_t render_symbol_sets(const uint32_t *sets, size_t n, char *out) {
    size_t o = 0;
    for (size_t i = 0; i < n; i++) {
        if (sets[i] == ORC_ALL) {
            out[o++] = '?';
        } else if ((sets[i] & (sets[i] - 1)) == 0) {
            out[o++] = B32[__builtin_ctz(sets[i])];
        } else {
            out[o++] = '[';
            for (int v = 0; v < 32; v++)
                if ((sets[i] >> v) & 1) out[o++] = B32[v];
            out[o++] = ']';
        }
    }
    out[o] = 0;
    return o;
}

static int parse_suffix_body(const char *s, size_t len, osuffix *out, char *err, size_t errlen) {
    size_t a = 0, b = len;
    while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) a++;
    while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) b--;
    memset(out, 0, sizeof *out);
    size_t n = 0;
    if (parse_symbol_body(s, a, b, out->sets, &n, err, errlen) != 0) return -1;
    if (n == 0) { snprintf(err, errlen, "empty"); return -1; }
    int fixed = 0;
    for (size_t i = 0; i < n; i++) fixed |= out->sets[i] != ORC_ALL;
    if (!fixed) { snprintf(err, errlen, "nothing fixed"); return -1; }
    if (!((out->sets[n - 1] >> symbol_value('d')) & 1)) { snprintf(err, errlen, "unreachable tail: last"); return -1; }
    if (n >= 2) {
        uint32_t tail = (1u << symbol_value('a')) | (1u << symbol_value('i')) | (1u << symbol_value('q')) |
                        (1u << symbol_value('y'));
        if (!(out->sets[n - 2] & tail)) { snprintf(err, errlen, "unreachable tail: penultimate"); return -1; }
    }
    out->len = n;
    /* a text key for sorting and de-duplication */
    render_symbol_sets(out->sets, n, out->text);
    return 0;
}

static int cmp_suffix(const void *x, const void *y) {
    return strcmp(((const osuffix *)x)->text, ((const osuffix *)y)->text);
}

/* suffix_slots (src/filter.rs:2438-2480): every slot of the window
 * [255 - bits, 255) the suffix allows, built symbol by symbol; 0 when more
 * than 4096. Returns the count, the slots in *out (malloc'd). */
static size_t suffix_slot_list(const osuffix *p, uint32_t bits, uint32_t **out) {
    size_t lo_bit = 255 - bits, hi_bit = 255, start = 56 - p->len;
    uint32_t *vals = malloc(sizeof *vals);
    size_t nv = 1;
    vals[0] = 0;
    for (size_t sym = lo_bit / 5; sym <= (hi_bit - 1) / 5; sym++) {
        size_t lo = sym * 5 > lo_bit ? sym * 5 : lo_bit;
        size_t hi = sym * 5 + 5 < hi_bit ? sym * 5 + 5 : hi_bit;
        size_t width = hi - lo, shift = hi_bit - hi;
        uint32_t set = sym >= start ? p->sets[sym - start] : ORC_ALL;
        if (sym == 49) set = orc_either_sign(set);
        uint32_t parts = 0; /* bitset of distinct parts (width <= 5) */
        for (unsigned v = 0; v < 32; v++)
            if ((set >> v) & 1) parts |= 1u << ((v >> (5 - (hi - sym * 5))) & ((1u << width) - 1));
        size_t np = (size_t)__builtin_popcount(parts);
        if (nv * np > 4096) {
            free(vals);
            *out = NULL;
            return 0;
        }
        uint32_t *next = malloc(nv * np * sizeof *next);
        size_t k = 0;
        for (size_t i = 0; i < nv; i++)
            for (unsigned part = 0; part < 32; part++)
                if ((parts >> part) & 1) next[k++] = vals[i] | (part << shift);
        free(vals);
        vals = next;
        nv = k;
    }
    *out = vals;
    return nv;
}

static uint64_t *suffix_map(const osuffix *p, size_t n, uint32_t bits, size_t *nwords) {
    size_t nw = (size_t)(((1ULL << bits) + 63) / 64);
    uint64_t *w = calloc(nw, sizeof *w);
    for (size_t i = 0; i < n; i++) {
        uint32_t *sl;
        size_t k = suffix_slot_list(&p[i], bits, &sl);
        if (!k) {
            free(w);
            return NULL;
        }
        for (size_t j = 0; j < k; j++) w[sl[j] >> 6] |= 1ULL << (sl[j] & 63);
        free(sl);
    }
    if (words_occupancy(w, nw, bits) > 0.25) {
        free(w);
        return NULL;
    }
    *nwords = nw;
    return w;
}

orc_sset *orc_sset_new(const char *text, uint32_t bits, char *err, size_t errlen) {
    size_t cap = 8, n = 0;
    osuffix *p = malloc(cap * sizeof *p);
    const char *q = text;
    while (*q) {
        const char *e = strchr(q, '\n');
        size_t len = e ? (size_t)(e - q) : strlen(q);
        int blank = 1;
        for (size_t i = 0; i < len; i++)
            if (q[i] != ' ' && q[i] != '\t' && q[i] != '\r') blank = 0;
        if (!blank) {
            if (n == cap) p = realloc(p, (cap *= 2) * sizeof *p);
            if (parse_suffix_body(q, len, &p[n], err, errlen) != 0) {
                free(p);
                return NULL;
            }
            n++;
        }
        if (!e) break;
        q = e + 1;
    }
    qsort(p, n, sizeof *p, cmp_suffix);
    size_t kept = 0;
    for (size_t i = 0; i < n; i++)
        if (!kept || strcmp(p[i].text, p[kept - 1].text) != 0) p[kept++] = p[i];
    orc_sset *s = calloc(1, sizeof *s);
    s->p = p;
    s->n = kept;
    if (bits == 0) {
        /* narrowest_acceptable(target_for_walk(n)) (src/filter.rs:2279-2300) */
        double target = 0.01 / (double)(kept ? kept : 1);
        for (uint32_t b = 16; b <= 24; b++) {
            size_t nw;
            uint64_t *w = suffix_map(p, kept, b, &nw);
            if (!w) continue;
            free(s->words);
            s->words = w;
            s->nwords = nw;
            s->bits = b;
            if (words_occupancy(w, nw, b) <= target) break;
        }
    } else {
        s->words = suffix_map(p, kept, bits, &s->nwords);
        s->bits = s->words ? bits : 0;
    }
    if (!s->words) {
        snprintf(err, errlen, "no suffix index could be built");
        orc_sset_free(s);
        return NULL;
    }
    return s;
}

void orc_sset_free(orc_sset *s) {
    if (!s) return;
    free(s->p);
    free(s->words);
    free(s);
}
size_t orc_sset_count(const orc_sset *s) { return s->n; }
uint32_t orc_sset_bits(const orc_sset *s) { return s->bits; }
size_t orc_sset_nwords(const orc_sset *s) { return s->nwords; }
const uint64_t *orc_sset_words(const orc_sset *s) { return s->words; }

/* BitmapIndex::slot with offset 255 - bits (src/filter.rs:2536-2549). */
int orc_sset_may_match(const orc_sset *s, const uint8_t packed[32]) {
    uint32_t slot = 0;
    for (uint32_t k = 0; k < s->bits; k++) {
        uint32_t bit = 255 - s->bits + k;
        slot = (slot << 1) | ((packed[bit / 8] >> (7 - bit % 8)) & 1);
    }
    return (int)((s->words[slot >> 6] >> (slot & 63)) & 1);
}

/* Filter::key_prefilter for a suffix (src/filter.rs:782-806). */
int orc_sset_key_prefilter(const orc_sset *s, size_t i, const uint8_t packed[32]) {
    const osuffix *p = &s->p[i];
    size_t start = 56 - p->len;
    for (size_t k = 0; k < p->len && start + k < 51; k++) {
        uint32_t set = start + k == 49 ? orc_either_sign(p->sets[k]) : p->sets[k];
        if (!((set >> orc_symbol_at(packed, 32, start + k)) & 1)) return 0;
    }
    return 1;
}

/* FilterSet::match_address over pk || checksum || 0x03 (src/filter.rs:2152). */
long orc_sset_match_pk(const orc_sset *s, const uint8_t pk[32]) {
    uint8_t a[35];
    memcpy(a, pk, 32);
    orc_checksum(pk, a + 32);
    a[34] = 0x03;
    for (size_t i = 0; i < s->n; i++) {
        const osuffix *p = &s->p[i];
        size_t start = 56 - p->len, k;
        for (k = 0; k < p->len; k++)
            if (!((p->sets[k] >> orc_symbol_at(a, 35, start + k)) & 1)) break;
        if (k == p->len) return (long)i;
    }
    return -1;
}
