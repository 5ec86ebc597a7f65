// Key-search kernels for sm_100a. See kernels.cuh for the schemes and the
// candidate numbering; field.cuh for the arithmetic.
#include "field.cuh"
#include "kernels.cuh"

// Register budget of the search kernels: at most OG_LB_THREADS threads per
// block and at least OG_LB_MIN_BLOCKS resident blocks per SM. 128 x 6 caps
// them at 80 registers (24 warps per SM), measured fastest on B200 against
// 96 (20 warps), 128 (16) and 130 registers.
#ifndef OG_LB_THREADS
#define OG_LB_THREADS 128
#endif
#ifndef OG_LB_MIN_BLOCKS
#define OG_LB_MIN_BLOCKS 6
#endif

namespace og {

namespace {

constexpr unsigned FULL = 0xffffffffu;

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

// Where survivors go: the bitmap, the record buffer and its counter.
struct Sink {
    const uint32_t* bitmap;
    uint32_t bits;
    HitRec* hits;
    uint32_t* counter;
    uint32_t cap;
    uint32_t search;
};

// Canonicalises y, tests its slot in the prefix bitmap and appends a record
// for every lane of the warp that hit, with one atomic per warp. Every lane
// of the warp must call this together (the kernels keep warps converged:
// lane counts are whole blocks and loop trip counts are uniform).
__device__ __forceinline__ void test_emit(const Sink& k, const fe& yraw, uint32_t lane, uint32_t step) {
    const fe y = fe_canon(yraw);
    bool hit = true;
    if (k.bitmap) {
        // bytes 0..3 of the key, big-endian: the top of the slot
        const uint32_t head = __byte_perm(y.v[0], 0, 0x0123);
        const uint32_t slot = k.bits >= 32 ? head : head >> (32 - k.bits);
        hit = (__ldg(k.bitmap + (slot >> 5)) >> (slot & 31)) & 1u;
    }
    const unsigned mask = __ballot_sync(FULL, hit);
    if (mask == 0) return;
    const unsigned me = threadIdx.x & 31u;
    const unsigned leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (me == leader) base = atomicAdd(k.counter, (uint32_t)__popc(mask));
    base = __shfl_sync(FULL, base, leader);
    if (hit) {
        const uint32_t idx = base + (uint32_t)__popc(mask & ((1u << me) - 1u));
        if (idx < k.cap) {
            uint4* rec = reinterpret_cast<uint4*>(k.hits + idx);
            rec[0] = make_uint4(lane, step, k.search, 0u);
            rec[1] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
            rec[2] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
        }
    }
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

__global__ void __launch_bounds__(128) init_kernel(const InitArgs a) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= a.lanes_n) return;
    const size_t L = a.lanes_n;
    fe X = words_fe(a.bx), Y = words_fe(a.by), Z = words_fe(a.bz), T = words_fe(a.bt);
    for (uint32_t k = 0; k < a.nbits; k++) {
        if ((lane >> k) & 1u) {
            const uint4* p = a.pow2 + (size_t)k * 6;
            const fe ypx = load_fe(p + 0, 1), ymx = load_fe(p + 2, 1), t2d = load_fe(p + 4, 1);
            add_cached(X, Y, Z, T, ypx, ymx, t2d);
        }
    }
    if (a.affine_out) {
        const fe zi = fe_invert(Z);
        store_fe(a.lanes + 0 * L + lane, L, fe_mulv(X, zi));
        store_fe(a.lanes + 2 * L + lane, L, fe_mulv(Y, zi));
    } else {
        store_fe(a.lanes + 0 * L + lane, L, X);
        store_fe(a.lanes + 2 * L + lane, L, Y);
        store_fe(a.lanes + 4 * L + lane, L, Z);
        store_fe(a.lanes + 6 * L + lane, L, T);
    }
}

__global__ void __launch_bounds__(OG_LB_THREADS, OG_LB_MIN_BLOCKS) paired_kernel(const PairedArgs a) {
    extern __shared__ uint4 qtab[];
    for (uint32_t i = threadIdx.x; i < a.half * 6; i += blockDim.x) qtab[i] = a.table[i];
    __syncthreads();

    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t L = a.lanes_n;
    const Sink sink{a.bitmap, a.bits, a.hits, a.counter, a.cap, a.search};
    const fe wx = words_fe(a.wx), wy = words_fe(a.wy), wt = words_fe(a.wt);
    const uint32_t half = a.half, slots = 2 * half + 1;
    uint4* const scr = a.scratch + lane;
    // scratch element e, part w (0 numerator, 1 denominator)
#define SCR(e, w) (scr + ((size_t)(e) * 4 + (w) * 2) * L)

    fe x = load_fe(a.lanes + 0 * L + lane, L);
    fe y = load_fe(a.lanes + 2 * L + lane, L);

    for (uint32_t r = 0; r < a.rounds; r++) {
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
#pragma unroll 1
        for (uint32_t m = 1; m <= half; m++) {
            const uint4* q = qtab + (size_t)(m - 1) * 6;
            const fe qx = load_fe(q + 0, 1), qy = load_fe(q + 2, 1), qt = load_fe(q + 4, 1);
            const fe A = fe_mulv(x, qy);
            const fe B = fe_mulv(y, qx);
            const fe d0 = fe_sub(A, B);  // P + Q_m
            store_fe(SCR(2 * m, 0), L, fe_mulv(fe_sub(t, qt), run));
            store_fe(SCR(2 * m, 1), L, d0);
            run = fe_mulv(run, d0);
            const fe d1 = fe_add(A, B);  // P - Q_m
            store_fe(SCR(2 * m + 1, 0), L, fe_mulv(fe_add(t, qt), run));
            store_fe(SCR(2 * m + 1, 1), L, d1);
            run = fe_mulv(run, d1);
        }
        fe acc = fe_invert(run);
        const uint32_t base_step = r * slots;
        test_emit(sink, y, lane, base_step + half);
#pragma unroll 1
        for (uint32_t m = half; m >= 1; m--) {
            {
                const fe v = fe_mulv(load_fe(SCR(2 * m + 1, 0), L), acc);
                acc = fe_mulv(acc, load_fe(SCR(2 * m + 1, 1), L));
                test_emit(sink, v, lane, base_step + half - m);
            }
            {
                const fe v = fe_mulv(load_fe(SCR(2 * m, 0), L), acc);
                acc = fe_mulv(acc, load_fe(SCR(2 * m, 1), L));
                test_emit(sink, v, lane, base_step + half + m);
            }
        }
        const fe xn = fe_mulv(load_fe(SCR(1, 0), L), acc);
        acc = fe_mulv(acc, load_fe(SCR(1, 1), L));
        y = fe_mulv(load_fe(SCR(0, 0), L), acc);
        x = xn;
    }
#undef SCR
    store_fe(a.lanes + 0 * L + lane, L, x);
    store_fe(a.lanes + 2 * L + lane, L, y);
}

// the chain kernel (parity contract, not the production path) keeps 96 registers: at 80 it spills
__global__ void __launch_bounds__(OG_LB_THREADS, 5) chain_kernel(const ChainArgs a) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t L = a.lanes_n;
    const Sink sink{a.bitmap, a.bits, a.hits, a.counter, a.cap, a.search};
    uint4* const scr = a.scratch + lane;
#define SCR(e, w) (scr + ((size_t)(e) * 4 + (w) * 2) * L)
    fe X = load_fe(a.lanes + 0 * L + lane, L);
    fe Y = load_fe(a.lanes + 2 * L + lane, L);
    fe Z = load_fe(a.lanes + 4 * L + lane, L);
    fe T = load_fe(a.lanes + 6 * L + lane, L);
    const fe sp = words_fe(a.step_ypx), sm = words_fe(a.step_ymx), st = words_fe(a.step_t2d);
    for (uint32_t r = 0; r < a.rounds; r++) {
        fe run = fe_one();
#pragma unroll 1
        for (uint32_t t = 0; t < a.n; t++) {
            store_fe(SCR(t, 0), L, fe_mulv(Y, run));
            store_fe(SCR(t, 1), L, Z);
            run = fe_mulv(run, Z);
            add_cached(X, Y, Z, T, sp, sm, st);
        }
        if (L > 1) add_cached(X, Y, Z, T, words_fe(a.jump_ypx), words_fe(a.jump_ymx), words_fe(a.jump_t2d));
        fe acc = fe_invert(run);
        const uint32_t base_step = r * a.n;
#pragma unroll 1
        for (uint32_t t = a.n; t-- > 0;) {
            const fe v = fe_mulv(load_fe(SCR(t, 0), L), acc);
            acc = fe_mulv(acc, load_fe(SCR(t, 1), L));
            test_emit(sink, v, lane, base_step + t);
        }
    }
#undef SCR
    store_fe(a.lanes + 0 * L + lane, L, X);
    store_fe(a.lanes + 2 * L + lane, L, Y);
    store_fe(a.lanes + 4 * L + lane, L, Z);
    store_fe(a.lanes + 6 * L + lane, L, T);
}

}  // namespace

cudaError_t launch_init(const InitArgs& a, int block, cudaStream_t s) {
    const unsigned grid = (a.lanes_n + block - 1) / block;
    init_kernel<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_paired(const PairedArgs& a, int block, cudaStream_t s) {
    if (a.lanes_n % block != 0 || block % 32 != 0) return cudaErrorInvalidValue;
    const size_t smem = (size_t)a.half * 96;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(paired_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    paired_kernel<<<a.lanes_n / block, block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_chain(const ChainArgs& a, int block, cudaStream_t s) {
    if (a.lanes_n % block != 0 || block % 32 != 0) return cudaErrorInvalidValue;
    chain_kernel<<<a.lanes_n / block, block, 0, s>>>(a);
    return cudaGetLastError();
}

static cudaError_t info_of(const void* fn, int block, size_t smem, KernelInfo* info) {
    cudaFuncAttributes attr;
    cudaError_t e = cudaFuncGetAttributes(&attr, fn);
    if (e != cudaSuccess) return e;
    info->regs = attr.numRegs;
    info->max_threads = attr.maxThreadsPerBlock;
    info->local_bytes = attr.localSizeBytes;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&info->blocks_per_sm, fn, block, smem);
}

cudaError_t paired_info(int block, uint32_t half, KernelInfo* info) {
    const size_t smem = (size_t)half * 96;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(paired_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return info_of((const void*)paired_kernel, block, smem, info);
}

cudaError_t chain_info(int block, KernelInfo* info) { return info_of((const void*)chain_kernel, block, 0, info); }

}  // namespace og
