// Device building blocks shared by the single-search and the batched
// kernels: device-layout loads and stores, the survivor test and append, the
// cached point addition, and one lane's paired rounds.
#pragma once
#include "field.cuh"
#include "kernels.cuh"

namespace og {

constexpr unsigned FULL = 0xffffffffu;

#ifndef OG_LB_THREADS
#define OG_LB_THREADS 128  // the most threads a block of the search kernels has
#endif

__device__ __forceinline__ fe load_fe(const uint4* p, size_t qstride) {
    const uint4 a = p[0];
    const uint4 b = p[qstride];
    fe r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}

__device__ __forceinline__ void store_fe(uint4* p, size_t qstride, const fe& v) {
    p[0] = make_uint4(v.v[0], v.v[1], v.v[2], v.v[3]);
    p[qstride] = make_uint4(v.v[4], v.v[5], v.v[6], v.v[7]);
}

__device__ __forceinline__ fe words_fe(const FeWords& w) {
    fe r;
#pragma unroll
    for (int k = 0; k < 8; k++) r.v[k] = w.v[k];
    return r;
}

// Where survivors go: the bitmaps, the record buffer and its counter.
struct Sink {
    const uint32_t* bitmap;
    uint32_t bits;
    HitRec* hits;
    uint32_t* counter;
    uint32_t cap;
    uint32_t search;
    const uint32_t* sbitmap;  // suffix bitmap, or nullptr
    uint32_t sbits;
    // the prefix bitmap is read from the block's copy in shared memory
    // (og_bitmap_s, staged by the kernel), not through L1
    bool staged = false;
};

// Prefix bitmaps of at most this many bits (8 KiB) can be staged in shared
// memory by a kernel that sets Sink::staged.
constexpr uint32_t STAGED_BITMAP_BITS = 16;

// Slot of a canonical key in the suffix bitmap: base32 bits
// [255 - sbits, 255) of the packed key, i.e. bits 1..sbits of its last eight
// bytes read big-endian (BitmapIndex::slot with offset 255 - sbits,
// src/filter.rs:2536-2549). The sign bit (bit 7 of byte 31) is clear in the
// packed key and the bitmap holds both of its values.
__device__ __forceinline__ uint32_t suffix_slot(const fe& y, uint32_t sbits) {
    const uint32_t lo = __byte_perm(y.v[7], 0, 0x0123), hi = __byte_perm(y.v[6], 0, 0x0123);
    const uint32_t w = (lo >> 1) | (hi << 31);
    return sbits >= 32 ? w : w & ((1u << sbits) - 1u);
}

// Survivor records staged per warp in shared memory, for dense indexes: a
// warp collects up to STAGE_RECORDS records and writes them with one atomic
// on the counter, where the direct append pays one for every warp-step that
// carries a survivor (at config 3's 5 % survivors, four warp-steps in five).
constexpr uint32_t STAGE_RECORDS = 32;

struct WarpStage {
    uint4* recs;  // this warp's STAGE_RECORDS records, three uint4 each, in shared memory
    uint32_t n;   // records held; the same in every lane of the warp
};

// Writes a warp's staged records to the sink (all lanes of the warp call it
// together). Records past the sink's room are counted, not written, as in
// test_emit.
__device__ __forceinline__ void stage_flush(const Sink& k, WarpStage& st) {
    if (st.n == 0) return;
    __syncwarp();
    const unsigned me = threadIdx.x & 31u;
    uint32_t base = 0;
    if (me == 0) base = atomicAdd(k.counter, st.n);
    base = __shfl_sync(FULL, base, 0);
    if (me < st.n && base + me < k.cap) {
        uint4* dst = reinterpret_cast<uint4*>(k.hits + base + me);
        const uint4* src = st.recs + me * 3;
        dst[0] = src[0];
        dst[1] = src[1];
        dst[2] = src[2];
    }
    __syncwarp();
    st.n = 0;
}

// Canonicalises y, tests its slot in the prefix bitmap and in the suffix
// bitmap (either lets it through; with neither, every candidate survives)
// and appends a record for every lane of the warp that hit, with one atomic
// per warp; with `Staged`, into the warp's stage `st` instead (flushed when
// full, and by the kernel at the end of each work item). Every lane of the
// warp must call this together (the kernels keep warps converged: lane
// counts are whole blocks and loop trip counts are uniform).
template <bool Staged = false>
__device__ __forceinline__ void test_emit(const Sink& k, const fe& yraw, uint32_t lane, uint32_t step,
                                          WarpStage* st = nullptr) {
    // The canonical limbs the bitmaps read (0, 6 and 7), without the full
    // canonicalisation. Folding bit 255 adds 19 to limb 0; its carry reaches
    // limb 6 only through limbs 1..5 all ones, and the value can be p or
    // more only with limbs 1..6 all ones (a carry out of limb 0 leaves it
    // below 19, too small for that). Outside that case, which a uniform key
    // meets with probability 2^-160, the canonical limbs are these.
    fe y;
    y.v[0] = yraw.v[0] + ((yraw.v[7] >> 31) ? 19u : 0u);
    y.v[6] = yraw.v[6];
    y.v[7] = yraw.v[7] & 0x7fffffffu;
    if ((yraw.v[1] & yraw.v[2] & yraw.v[3] & yraw.v[4] & yraw.v[5]) == 0xffffffffu) y = fe_canon(yraw);
    bool hit = true;
    if (k.bitmap || k.sbitmap) {
        hit = false;
        if (k.bitmap) {
            // bytes 0..3 of the key, big-endian: the top of the slot
            const uint32_t head = __byte_perm(y.v[0], 0, 0x0123);
            const uint32_t slot = k.bits >= 32 ? head : head >> (32 - k.bits);
            if (k.staged) {
                extern __shared__ uint32_t og_bitmap_s[];
                hit = (og_bitmap_s[slot >> 5] >> (slot & 31)) & 1u;
            } else {
                hit = (__ldg(k.bitmap + (slot >> 5)) >> (slot & 31)) & 1u;
            }
        }
        if (k.sbitmap) {
            const uint32_t slot = suffix_slot(y, k.sbits);
            hit |= ((__ldg(k.sbitmap + (slot >> 5)) >> (slot & 31)) & 1u) != 0;
        }
    }
    const unsigned mask = __ballot_sync(FULL, hit);
    if (mask == 0) return;
    const unsigned me = threadIdx.x & 31u;
    if constexpr (Staged) {
        const uint32_t count = (uint32_t)__popc(mask);
        if (st->n + count > STAGE_RECORDS) stage_flush(k, *st);
        if (hit) {
            const uint32_t idx = st->n + (uint32_t)__popc(mask & ((1u << me) - 1u));
            y = fe_canon(yraw);
            uint4* rec = st->recs + idx * 3;
            rec[0] = make_uint4(lane, step, k.search, 0u);
            rec[1] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
            rec[2] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
        }
        st->n += count;
        return;
    }
    const unsigned leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (me == leader) base = atomicAdd(k.counter, (uint32_t)__popc(mask));
    base = __shfl_sync(FULL, base, leader);
    if (hit) {
        const uint32_t idx = base + (uint32_t)__popc(mask & ((1u << me) - 1u));
        if (idx < k.cap) {
            y = fe_canon(yraw);
            uint4* rec = reinterpret_cast<uint4*>(k.hits + idx);
            rec[0] = make_uint4(lane, step, k.search, 0u);
            rec[1] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
            rec[2] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
        }
    }
}

// Symbol `pos` (five bits, most significant first) of a canonical key held
// as eight little-endian limbs, i.e. of its 32 packed bytes.
__device__ __forceinline__ uint32_t key_symbol(const uint32_t y[8], uint32_t pos) {
    const uint32_t bit = pos * 5, byte = bit / 8;
    const uint32_t b0 = (y[byte / 4] >> (8 * (byte % 4))) & 0xffu;
    const uint32_t b1 = byte + 1 < 32 ? (y[(byte + 1) / 4] >> (8 * ((byte + 1) % 4))) & 0xffu : 0u;
    return (((b0 << 8) | b1) >> (11 - bit % 8)) & 31u;
}

// The filter a canonical key matches, or 0xffffffff: per length bucket of
// the literal prefixes a binary search of the sorted masked heads (first 12
// symbols at most; no kept literal is a prefix of another, so at most one
// matches), then the patterns in order, on their key-only symbols.
__device__ __forceinline__ uint32_t exact_owner(const MatchTables& t, const uint32_t y[8]) {
    const uint64_t head = ((uint64_t)__byte_perm(y[0], 0, 0x0123) << 32) | (uint64_t)__byte_perm(y[1], 0, 0x0123);
    for (uint32_t b = 0; b < t.nbuckets; b++) {
        const uint64_t probe = head & (~0ULL << (64 - t.bucket_bits[b]));
        const uint64_t* k = t.keys + t.bucket_off[b];
        uint32_t lo = 0, hi = t.bucket_len[b];
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (k[mid] < probe) lo = mid + 1;
            else hi = mid;
        }
        if (lo < t.bucket_len[b] && k[lo] == probe) return t.owners[t.bucket_off[b] + lo];
    }
    for (uint32_t j = 0; j < t.npatterns; j++) {
        const uint32_t* p = t.patterns + (size_t)j * PATTERN_WORDS;
        bool ok = true;
        for (uint32_t i = 0; i < p[1] && ok; i++) ok = (p[2 + i] >> key_symbol(y, i)) & 1u;
        if (ok) return p[0];
    }
    return 0xffffffffu;
}

__device__ __forceinline__ fe shfl_up_fe(const fe& v, unsigned d) {
    fe r;
#pragma unroll
    for (int k = 0; k < 8; k++) r.v[k] = __shfl_up_sync(FULL, v.v[k], d);
    return r;
}

__device__ __forceinline__ fe shfl_down_fe(const fe& v, unsigned d) {
    fe r;
#pragma unroll
    for (int k = 0; k < 8; k++) r.v[k] = __shfl_down_sync(FULL, v.v[k], d);
    return r;
}

__device__ __forceinline__ fe select_fe(bool c, const fe& a, const fe& b) {
    fe r;
#pragma unroll
    for (int k = 0; k < 8; k++) r.v[k] = c ? a.v[k] : b.v[k];
    return r;
}

// 1/v for every thread of the block with one field inversion for the whole
// block: Montgomery's trick across its lanes. A warp executes an inversion
// at the cost of all its lanes whether one lane or 32 need it, so one
// inversion a block instead of one a warp saves three of every four on
// 128-thread blocks. Within a warp, inclusive prefix and suffix products by
// shuffles (five levels each, the missing neighbours taken as 1); across
// warps, their totals in shared memory; thread 0 inverts the block's total;
// then 1/v_i = (product before i) (product after i) / total. The inverse is
// unique, so the result equals fe_invert's modulo p (0 when some v of the
// block is 0, which the search's denominators never are). Every thread of
// the block calls it together; blocks hold at most OG_LB_THREADS threads.
// Not inlined, like fe_invert, so that the search loops' register
// allocation does not change around it.
static __device__ __noinline__ fe block_invert(const fe& v) {
    __shared__ fe warp_total_s[OG_LB_THREADS / 32];
    __shared__ fe inv_total_s;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const fe one = fe_one();
    fe pre = v, suf = v;
#pragma unroll
    for (unsigned d = 1; d < 32; d <<= 1) {
        const fe lo = shfl_up_fe(pre, d), hi = shfl_down_fe(suf, d);
        pre = fe_mulv(pre, select_fe(lane >= d, lo, one));
        suf = fe_mulv(suf, select_fe(lane + d < 32, hi, one));
    }
    // exclusive: the products strictly before and after this lane
    const fe before = select_fe(lane > 0, shfl_up_fe(pre, 1), one);
    const fe after = select_fe(lane < 31, shfl_down_fe(suf, 1), one);
    __syncthreads();  // earlier readers of the shared words are done
    if (lane == 31) warp_total_s[warp] = pre;
    __syncthreads();
    if (threadIdx.x == 0) {
        fe total = warp_total_s[0];
        for (unsigned w = 1; w < nwarps; w++) total = fe_mulv(total, warp_total_s[w]);
        inv_total_s = fe_invert(total);
    }
    // the other warps' totals, before and after this warp (the same in every lane)
    fe others = one;
    for (unsigned w = 0; w < nwarps; w++)
        if (w != warp) others = fe_mulv(others, warp_total_s[w]);
    __syncthreads();
    return fe_mulv(fe_mulv(before, after), fe_mulv(others, inv_total_s));
}

// p3 + cached addend with Z = 1: seven multiplications
// (the formulas of src/curve.rs:130-175 with the addend's Z scaled away).
__device__ __forceinline__ void add_cached(fe& X, fe& Y, fe& Z, fe& T, const fe& ypx, const fe& ymx,
                                           const fe& t2d) {
    const fe a = fe_mulv(fe_add(Y, X), ypx);
    const fe b = fe_mulv(fe_sub(Y, X), ymx);
    const fe c = fe_mulv(T, t2d);
    const fe d = fe_add(Z, Z);
    const fe x3 = fe_sub(a, b), y3 = fe_add(a, b), z3 = fe_add(d, c), t3 = fe_sub(d, c);
    X = fe_mulv(x3, t3);
    Y = fe_mulv(y3, z3);
    Z = fe_mulv(z3, t3);
    T = fe_mulv(x3, y3);
}

// A lane's centre x, y and t = x y parked in shared memory for the forward
// pass: each fe as two 16-byte quarters at park[(k * 2 + q) * PARK_STRIDE],
// so a warp's loads are conflict-free. Loaded with volatile asm right
// before each use so that the compiler cannot hoist them back into
// registers for the whole loop. The 24 registers this frees took the
// single-search kernel at 96 registers from 72 bytes of spills to 4 and
// from 20.6 to 20.8 G keys/s on B200. The batched kernel does not park
// (Park = false): with its staged bitmap the 12 KB a block would leave L1
// too small for the table Q_m at half 2048, and it ran 6 % slower parked.
constexpr int PARK_STRIDE = OG_LB_THREADS;

__device__ __forceinline__ void park_fe(uint4* park, int k, const fe& v) {
    park[(k * 2 + 0) * PARK_STRIDE] = make_uint4(v.v[0], v.v[1], v.v[2], v.v[3]);
    park[(k * 2 + 1) * PARK_STRIDE] = make_uint4(v.v[4], v.v[5], v.v[6], v.v[7]);
}

__device__ __forceinline__ fe unpark_fe(const uint4* park, int k) {
    fe r;
    const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(park + (k * 2 + 0) * PARK_STRIDE);
    const uint32_t a1 = (uint32_t)__cvta_generic_to_shared(park + (k * 2 + 1) * PARK_STRIDE);
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]) : "r"(a0));
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]), "=r"(r.v[7]) : "r"(a1));
    return r;
}

// One lane's `rounds` paired rounds around its affine centre (x, y); see
// kernels.cuh for the formulas and the candidate numbering. `scr` is the
// lane's scratch: element e, part w (0 numerator, 1 denominator), half q at
// scr + ((e * 2 + w) * 2 + q) * stride. `visit(y, step)` receives every
// candidate's y (not yet canonical) with step = round * (2 half + 1) + index.
// Park: keep the centre in shared memory during the forward pass (above).
template <bool Park, class Visit>
__device__ __forceinline__ void paired_rounds(fe& x, fe& y, const fe& wx, const fe& wy, const fe& wt,
                                              const uint4* qtab, uint32_t half, uint32_t rounds, uint4* scr,
                                              size_t stride, Visit&& visit) {
    const size_t L = stride;
    const uint32_t slots = 2 * half + 1;
    __shared__ uint4 park_s[Park ? 6 * PARK_STRIDE : 1];
    uint4* const park = park_s + (Park ? threadIdx.x : 0);
#define SCR(e, w) (scr + ((size_t)(e) * 4 + (w) * 2) * L)
    for (uint32_t r = 0; r < rounds; r++) {
        const fe t = fe_mulv(x, y);
        // e = 0: y(P + W) = (t - tW) / (x yW - y xW); e = 1: x(P + W) = (t + tW) / (y yW - x xW)
        fe run;
        {
            const fe den0 = fe_sub(fe_mulv(x, wy), fe_mulv(y, wx));
            store_fe(SCR(0, 0), L, fe_sub(t, wt));
            store_fe(SCR(0, 1), L, den0);
            const fe den1 = fe_sub(fe_mulv(y, wy), fe_mulv(x, wx));
            store_fe(SCR(1, 0), L, fe_mulv(fe_add(t, wt), den0));
            store_fe(SCR(1, 1), L, den1);
            run = fe_mulv(den0, den1);
        }
        if (Park) {
            park_fe(park, 0, x);
            park_fe(park, 1, y);
            park_fe(park, 2, t);
        }
        const auto centre = [&](int k) -> fe { return Park ? unpark_fe(park, k) : k == 0 ? x : k == 1 ? y : t; };
#pragma unroll 1
        for (uint32_t m = 1; m <= half; m++) {
            const uint4* q = qtab + (size_t)(m - 1) * 6;
            const fe A = fe_mulv(centre(0), load_fe(q + 2, 1));
            const fe B = fe_mulv(centre(1), load_fe(q + 0, 1));
            const fe d0 = fe_sub(A, B);  // P + Q_m
            const fe qt = load_fe(q + 4, 1);
            store_fe(SCR(2 * m, 0), L, fe_mulv(fe_sub(centre(2), qt), run));
            store_fe(SCR(2 * m, 1), L, d0);
            run = fe_mulv(run, d0);
            const fe d1 = fe_add(A, B);  // P - Q_m
            store_fe(SCR(2 * m + 1, 0), L, fe_mulv(fe_add(centre(2), qt), run));
            store_fe(SCR(2 * m + 1, 1), L, d1);
            run = fe_mulv(run, d1);
        }
        // one inversion for the block's lanes where the centre is parked; the
        // batched kernel keeps it in registers, which the call would save and
        // restore (measured 1 % slower there), so it inverts per lane
        fe acc = Park ? block_invert(run) : fe_invert(run);
        const uint32_t base_step = r * slots;
        visit(centre(1), base_step + half);
#pragma unroll 1
        for (uint32_t m = half; m >= 1; m--) {
            {
                const fe v = fe_mulv(load_fe(SCR(2 * m + 1, 0), L), acc);
                acc = fe_mulv(acc, load_fe(SCR(2 * m + 1, 1), L));
                visit(v, base_step + half - m);
            }
            {
                const fe v = fe_mulv(load_fe(SCR(2 * m, 0), L), acc);
                acc = fe_mulv(acc, load_fe(SCR(2 * m, 1), L));
                visit(v, base_step + half + m);
            }
        }
        const fe xn = fe_mulv(load_fe(SCR(1, 0), L), acc);
        acc = fe_mulv(acc, load_fe(SCR(1, 1), L));
        y = fe_mulv(load_fe(SCR(0, 0), L), acc);
        x = xn;
    }
#undef SCR
}

// N lanes per thread (N = 2): the rounds of paired_rounds for the lanes
// (x[k], y[k]), k < N, whose scratch columns start at scr[k] (element e,
// part w, half q at scr[k] + ((e * 2 + w) * 2 + q) * stride). The lanes'
// passes are written step by step side by side, so that the scheduler can
// issue one lane's products while the other lane's carry chains settle, and
// the lanes of a thread share the table loads and one inversion per round
// (Montgomery's trick over their N final products: 1 inversion and 3
// multiplications instead of 2 inversions). `visit(k, y, step)` receives
// lane k's candidates with the numbering of paired_rounds. Centres are
// parked in shared memory as there (3 N field elements a thread).
template <int N, class Visit>
__device__ __forceinline__ void paired_rounds_n(fe (&x)[N], fe (&y)[N], const fe& wx, const fe& wy, const fe& wt,
                                                const uint4* qtab, uint32_t half, uint32_t rounds,
                                                uint4* const (&scr)[N], size_t stride, Visit&& visit) {
    static_assert(N == 2, "paired_rounds covers one lane a thread; this function two");
    const size_t L = stride;
    const uint32_t slots = 2 * half + 1;
    __shared__ uint4 park_s[N * 6 * PARK_STRIDE];
    uint4* const park = park_s + threadIdx.x;
#define SCRN(k, e, w) (scr[k] + ((size_t)(e) * 4 + (w) * 2) * L)
    for (uint32_t r = 0; r < rounds; r++) {
        fe run[N];
#pragma unroll
        for (int k = 0; k < N; k++) {
            const fe t = fe_mulv(x[k], y[k]);
            const fe den0 = fe_sub(fe_mulv(x[k], wy), fe_mulv(y[k], wx));
            store_fe(SCRN(k, 0, 0), L, fe_sub(t, wt));
            store_fe(SCRN(k, 0, 1), L, den0);
            const fe den1 = fe_sub(fe_mulv(y[k], wy), fe_mulv(x[k], wx));
            store_fe(SCRN(k, 1, 0), L, fe_mulv(fe_add(t, wt), den0));
            store_fe(SCRN(k, 1, 1), L, den1);
            run[k] = fe_mulv(den0, den1);
            park_fe(park, 3 * k + 0, x[k]);
            park_fe(park, 3 * k + 1, y[k]);
            park_fe(park, 3 * k + 2, t);
        }
#pragma unroll 1
        for (uint32_t m = 1; m <= half; m++) {
            const uint4* q = qtab + (size_t)(m - 1) * 6;
            fe A[N], B[N];
#pragma unroll
            for (int k = 0; k < N; k++) {
                A[k] = fe_mulv(unpark_fe(park, 3 * k + 0), load_fe(q + 2, 1));
                B[k] = fe_mulv(unpark_fe(park, 3 * k + 1), load_fe(q + 0, 1));
            }
            const fe qt = load_fe(q + 4, 1);
#pragma unroll
            for (int k = 0; k < N; k++) {
                const fe d0 = fe_sub(A[k], B[k]);  // P + Q_m
                const fe tk = unpark_fe(park, 3 * k + 2);
                store_fe(SCRN(k, 2 * m, 0), L, fe_mulv(fe_sub(tk, qt), run[k]));
                store_fe(SCRN(k, 2 * m, 1), L, d0);
                run[k] = fe_mulv(run[k], d0);
                const fe d1 = fe_add(A[k], B[k]);  // P - Q_m
                store_fe(SCRN(k, 2 * m + 1, 0), L, fe_mulv(fe_add(tk, qt), run[k]));
                store_fe(SCRN(k, 2 * m + 1, 1), L, d1);
                run[k] = fe_mulv(run[k], d1);
            }
        }
        fe acc[N];
        {
            const fe inv = fe_invert(fe_mulv(run[0], run[1]));
            acc[0] = fe_mulv(inv, run[1]);
            acc[1] = fe_mulv(inv, run[0]);
        }
        const uint32_t base_step = r * slots;
#pragma unroll
        for (int k = 0; k < N; k++) visit(k, unpark_fe(park, 3 * k + 1), base_step + half);
#pragma unroll 1
        for (uint32_t m = half; m >= 1; m--) {
            fe v[N];
#pragma unroll
            for (int k = 0; k < N; k++) {
                v[k] = fe_mulv(load_fe(SCRN(k, 2 * m + 1, 0), L), acc[k]);
                acc[k] = fe_mulv(acc[k], load_fe(SCRN(k, 2 * m + 1, 1), L));
            }
#pragma unroll
            for (int k = 0; k < N; k++) visit(k, v[k], base_step + half - m);
#pragma unroll
            for (int k = 0; k < N; k++) {
                v[k] = fe_mulv(load_fe(SCRN(k, 2 * m, 0), L), acc[k]);
                acc[k] = fe_mulv(acc[k], load_fe(SCRN(k, 2 * m, 1), L));
            }
#pragma unroll
            for (int k = 0; k < N; k++) visit(k, v[k], base_step + half + m);
        }
#pragma unroll
        for (int k = 0; k < N; k++) {
            const fe xn = fe_mulv(load_fe(SCRN(k, 1, 0), L), acc[k]);
            acc[k] = fe_mulv(acc[k], load_fe(SCRN(k, 1, 1), L));
            y[k] = fe_mulv(load_fe(SCRN(k, 0, 0), L), acc[k]);
            x[k] = xn;
        }
    }
#undef SCRN
}

}  // namespace og
