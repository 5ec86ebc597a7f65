// GF(2^255-19) on sm_100a: eight 32-bit limbs, least significant first.
//
// Every value is held below 2^256 and congruent to the field element; only
// fe_canon() produces the unique representative below p. Multiplication and
// squaring are exact 32x32->64 partial products on the integer multiply-add
// pipe with PTX carry chains (field_asm.cuh); addition and subtraction are
// carry chains on the integer ALU, folded with 2^256 = 38 (mod p).
//
// The representation and folding constant follow the arithmetic of
// src/field.rs (radix 2^64 there, radix 2^32 here) and the device field of
// cuda-kernel/src/field_asm.rs; the code is written for this engine.
#pragma once
#include <cstdint>

#include "field_asm.cuh"

struct fe {
    uint32_t v[8];
};

#define OG_FE_MUL_ASM fe_mul_asm

__device__ __forceinline__ void fe_mul(fe& r, const fe& a, const fe& b) { OG_FE_MUL_ASM(r.v, a.v, b.v); }
__device__ __forceinline__ void fe_sq(fe& r, const fe& a) { fe_sq_asm(r.v, a.v); }

__device__ __forceinline__ fe fe_mulv(const fe& a, const fe& b) {
    fe r;
    OG_FE_MUL_ASM(r.v, a.v, b.v);
    return r;
}

__device__ __forceinline__ fe fe_sqv(const fe& a) {
    fe r;
    fe_sq_asm(r.v, a.v);
    return r;
}

// r = a + b. A carry out of bit 256 is worth 38; a second fold cannot carry.
__device__ __forceinline__ fe fe_add(const fe& a, const fe& b) {
    fe r;
    asm("{\n\t.reg .u32 c, m;\n\t"
        "add.cc.u32 %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.cc.u32 %7, %15, %23;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 m, c;\n\t"
        "and.b32 m, m, 38;\n\t"
        "add.cc.u32 %0, %0, m;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.cc.u32 %4, %4, 0;\n\t"
        "addc.cc.u32 %5, %5, 0;\n\t"
        "addc.cc.u32 %6, %6, 0;\n\t"
        "addc.cc.u32 %7, %7, 0;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 m, c;\n\t"
        "and.b32 m, m, 38;\n\t"
        "add.u32 %0, %0, m;\n\t"
        "}"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
          "=r"(r.v[6]), "=r"(r.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
          "r"(b.v[6]), "r"(b.v[7]));
    return r;
}

// r = a - b. A borrow out of the top means the value wrapped by 2^256, which
// is worth 38, so 38 is taken off again; a second borrow leaves the value near
// 2^256 and the third subtraction cannot borrow.
__device__ __forceinline__ fe fe_sub(const fe& a, const fe& b) {
    fe r;
    asm("{\n\t.reg .u32 c, m;\n\t"
        "sub.cc.u32 %0, %8, %16;\n\t"
        "subc.cc.u32 %1, %9, %17;\n\t"
        "subc.cc.u32 %2, %10, %18;\n\t"
        "subc.cc.u32 %3, %11, %19;\n\t"
        "subc.cc.u32 %4, %12, %20;\n\t"
        "subc.cc.u32 %5, %13, %21;\n\t"
        "subc.cc.u32 %6, %14, %22;\n\t"
        "subc.cc.u32 %7, %15, %23;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "and.b32 m, c, 38;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.cc.u32 %2, %2, 0;\n\t"
        "subc.cc.u32 %3, %3, 0;\n\t"
        "subc.cc.u32 %4, %4, 0;\n\t"
        "subc.cc.u32 %5, %5, 0;\n\t"
        "subc.cc.u32 %6, %6, 0;\n\t"
        "subc.cc.u32 %7, %7, 0;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "and.b32 m, c, 38;\n\t"
        "sub.u32 %0, %0, m;\n\t"
        "}"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
          "=r"(r.v[6]), "=r"(r.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
          "r"(b.v[6]), "r"(b.v[7]));
    return r;
}

// a + c for a small c, carried through all limbs; the caller guarantees
// that the sum stays below 2^256.
__device__ __forceinline__ fe fe_add_small(const fe& a, uint32_t c) {
    fe r;
    asm("add.cc.u32 %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, 0;\n\t"
        "addc.cc.u32 %2, %10, 0;\n\t"
        "addc.cc.u32 %3, %11, 0;\n\t"
        "addc.cc.u32 %4, %12, 0;\n\t"
        "addc.cc.u32 %5, %13, 0;\n\t"
        "addc.cc.u32 %6, %14, 0;\n\t"
        "addc.u32 %7, %15, 0;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
          "=r"(r.v[6]), "=r"(r.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(c));
    return r;
}

// The unique representative below p = 2^255 - 19.
// Bit 255 is folded first (2^255 = 19), which leaves a value below
// 2^255 + 19; then q = (v + 19) >> 255 says whether one p comes off, and
// v - q p = (v + 19 q) mod 2^255.
__device__ __forceinline__ fe fe_canon(const fe& a) {
    fe v = a;
    const uint32_t top = v.v[7] >> 31;
    v.v[7] &= 0x7fffffffu;
    v = fe_add_small(v, top * 19u);
    fe s = fe_add_small(v, 19u);
    const bool q = (s.v[7] >> 31) != 0;
    s.v[7] &= 0x7fffffffu;
    fe r;
#pragma unroll
    for (int k = 0; k < 8; k++) r.v[k] = q ? s.v[k] : v.v[k];
    return r;
}

__device__ __forceinline__ fe fe_one() {
    fe r;
#pragma unroll
    for (int k = 0; k < 8; k++) r.v[k] = k == 0 ? 1u : 0u;
    return r;
}

__device__ __forceinline__ fe fe_sqn(fe a, int n) {
#pragma unroll 1
    for (int i = 0; i < n; i++) a = fe_sqv(a);
    return a;
}

// x^(p-2) = x^-1 (and 0 for 0). The addition chain is the standard one for
// 2^255 - 21: it builds x^(2^k - 1) for k = 5, 10, 20, 40, 50, 100, 200, 250
// by squaring runs and multiplications, then 2^255 - 21 = (2^250 - 1) 2^5 + 11.
// 254 squarings and 11 multiplications.
static __device__ __noinline__ fe fe_invert(const fe& z) {
    const fe z2 = fe_sqv(z);                       // 2
    const fe z9 = fe_mulv(fe_sqv(fe_sqv(z2)), z);  // 9
    const fe z11 = fe_mulv(z9, z2);                // 11
    const fe e5 = fe_mulv(fe_sqv(z11), z9);        // 2^5 - 1
    const fe e10 = fe_mulv(fe_sqn(e5, 5), e5);     // 2^10 - 1
    const fe e20 = fe_mulv(fe_sqn(e10, 10), e10);  // 2^20 - 1
    const fe e40 = fe_mulv(fe_sqn(e20, 20), e20);  // 2^40 - 1
    const fe e50 = fe_mulv(fe_sqn(e40, 10), e10);  // 2^50 - 1
    const fe e100 = fe_mulv(fe_sqn(e50, 50), e50); // 2^100 - 1
    const fe e200 = fe_mulv(fe_sqn(e100, 100), e100);
    const fe e250 = fe_mulv(fe_sqn(e200, 50), e50);
    return fe_mulv(fe_sqn(e250, 5), z11);          // 2^255 - 21
}
