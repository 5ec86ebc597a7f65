// Key-search kernels for sm_100a. See kernels.cuh for the schemes and the
// candidate numbering; field.cuh for the arithmetic.
#include "field.cuh"
#include "kernels.cuh"
#include "search_common.cuh"
#include "suffix_match.cuh"

// Register budget of the search kernels: at most OG_LB_THREADS threads per
// block and at least OG_LB_MIN_BLOCKS resident blocks per SM. 128 x 5 caps
// them at 96 registers (20 warps per SM). With the two-accumulator field
// multiply this measured fastest on B200: 20.5 G keys/s against 20.0 at
// 80 registers (24 warps, more spills) and 20.3 at 128 (16 warps). With the
// lane's centre parked in shared memory (paired_rounds) it spills 4 bytes
// and runs 20.8; at 80 registers 20.9 at half 2048 but 20.7 at half 1024.
#ifndef OG_LB_THREADS
#define OG_LB_THREADS 128
#endif
#ifndef OG_LB_MIN_BLOCKS
#define OG_LB_MIN_BLOCKS 5
#endif

namespace og {

namespace {

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

// Staged: survivor records collected per warp in shared memory and written
// 32 at a time (WarpStage), for indexes that let many candidates through.
template <bool Staged>
__global__ void __launch_bounds__(OG_LB_THREADS, OG_LB_MIN_BLOCKS) paired_kernel(const PairedArgs a) {
    // The table is read through L1, not staged in shared memory: every lane
    // of a warp loads the same entry, and leaving shared memory unused keeps
    // large tables from capping occupancy (measured 17.97 vs 13.3 G keys/s
    // at half 1024, and the same speed at half 256).
    const uint4* qtab = a.table;
    // Persistent: each CTA takes the next block of lanes until none is left.
    // The scratch is indexed by the CTA's slot, not the lane.
    __shared__ uint32_t item_s;
    const size_t L = a.lanes_n, S = a.slots_n;
    const uint32_t nblocks = a.lanes_n / blockDim.x;
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const Sink sink{a.bitmap, a.bits, a.hits, a.counter, a.cap, a.search, a.sbitmap, a.sbits};
    __shared__ uint4 stage_s[Staged ? (OG_LB_THREADS / 32) * STAGE_RECORDS * 3 : 1];
    WarpStage st{stage_s + (Staged ? (threadIdx.x / 32) * STAGE_RECORDS * 3 : 0), 0};
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_s = atomicAdd(a.work, 1u);
        __syncthreads();
        const uint32_t item = item_s;
        if (item >= nblocks) break;
        const uint32_t lane = item * blockDim.x + threadIdx.x;
        fe x = load_fe(a.lanes + 0 * L + lane, L);
        fe y = load_fe(a.lanes + 2 * L + lane, L);
        paired_rounds<true>(x, y, words_fe(a.wx), words_fe(a.wy), words_fe(a.wt), qtab, a.half, a.rounds, a.scratch + slot, S,
                      [&](const fe& v, uint32_t step) { test_emit<Staged>(sink, v, lane, step, &st); });
        if (Staged) stage_flush(sink, st);
        store_fe(a.lanes + 0 * L + lane, L, x);
        store_fe(a.lanes + 2 * L + lane, L, y);
    }
}

// Two lanes per thread (paired_rounds_n): each work item is 2 blocks of
// lanes, thread t taking lanes item * 2 B + t and item * 2 B + B + t; the
// scratch has two columns per thread, slot t and slot t + S / 2. Its
// register bound (128 threads, OG_LB2_MIN_BLOCKS blocks per SM) holds the
// two lanes' field elements without spills.
#ifndef OG_LB2_MIN_BLOCKS
#define OG_LB2_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(OG_LB_THREADS, OG_LB2_MIN_BLOCKS) paired_kernel2(const PairedArgs a) {
    const uint4* qtab = a.table;
    __shared__ uint32_t item_s;
    const size_t L = a.lanes_n, S = a.slots_n;
    const uint32_t per_item = 2 * blockDim.x;
    const uint32_t nitems = a.lanes_n / per_item;
    const uint32_t half_slots = a.slots_n / 2;
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    uint4* const scr[2] = {a.scratch + slot, a.scratch + half_slots + slot};
    const Sink sink{a.bitmap, a.bits, a.hits, a.counter, a.cap, a.search, a.sbitmap, a.sbits};
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_s = atomicAdd(a.work, 1u);
        __syncthreads();
        const uint32_t item = item_s;
        if (item >= nitems) break;
        const uint32_t lane[2] = {item * per_item + threadIdx.x, item * per_item + blockDim.x + threadIdx.x};
        fe x[2], y[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            x[k] = load_fe(a.lanes + 0 * L + lane[k], L);
            y[k] = load_fe(a.lanes + 2 * L + lane[k], L);
        }
        paired_rounds_n<2>(x, y, words_fe(a.wx), words_fe(a.wy), words_fe(a.wt), qtab, a.half, a.rounds, scr, S,
                           [&](int k, const fe& v, uint32_t step) { test_emit(sink, v, lane[k], step); });
#pragma unroll
        for (int k = 0; k < 2; k++) {
            store_fe(a.lanes + 0 * L + lane[k], L, x[k]);
            store_fe(a.lanes + 2 * L + lane[k], L, y[k]);
        }
    }
}

// The chain kernel (the config-1 contract) keeps 96 registers: at 80 it
// spills. Persistent like the paired kernel: each CTA takes the next block
// of lanes until none is left, and the scratch is indexed by the CTA's
// slot, so any number of waves of lanes costs the scratch of one. A prefix
// bitmap of up to 16 bits (8 KiB) is staged in shared memory per CTA and
// tested there: 9.445e9 against 9.355e9 keys/s on B200 for config 2's index
// at n = 1024. (The paired kernel reads the table Q_m through L1, and the
// 8 KiB more a block cost it more than the bitmap read saves, so it keeps
// the map in global memory.) The scratch is one region per CTA whose rows
// hold the CTA's threads, so that a CTA's accesses stay within a few pages:
// 9.57e9 against 9.49e9 keys/s with rows across the whole grid.
__global__ void __launch_bounds__(OG_LB_THREADS, 5) chain_kernel(const ChainArgs a) {
    static_assert(CHAIN_ROW >= OG_LB_THREADS, "a row holds every thread of a block");
    __shared__ uint32_t item_s;
    const size_t L = a.lanes_n;
    const uint32_t nblocks = a.lanes_n / blockDim.x;
    const bool staged = a.bitmap && a.bits <= STAGED_BITMAP_BITS;
    const Sink sink{a.bitmap, a.bits, a.hits, a.counter, a.cap, a.search, a.sbitmap, a.sbits, staged};
    if (staged) {
        extern __shared__ uint32_t og_bitmap_s[];
        const uint32_t words = (1u << a.bits) / 32u;
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) og_bitmap_s[i] = a.bitmap[i];
        // the loop's first barrier orders these stores before any test
    }
    uint4* const scr = a.scratch + (size_t)blockIdx.x * (CHAIN_ROW * 4) * a.n + threadIdx.x;
#define SCR(e, w) (scr + ((size_t)(e) * 4 + (w) * 2) * CHAIN_ROW)
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_s = atomicAdd(a.work, 1u);
        __syncthreads();
        const uint32_t item = item_s;
        if (item >= nblocks) break;
        const uint32_t lane = item * blockDim.x + threadIdx.x;
        fe X = load_fe(a.lanes + 0 * L + lane, L);
        fe Y = load_fe(a.lanes + 2 * L + lane, L);
        fe Z = load_fe(a.lanes + 4 * L + lane, L);
        fe T = load_fe(a.lanes + 6 * L + lane, L);
        for (uint32_t r = 0; r < a.rounds; r++) {
            fe run = fe_one();
#pragma unroll 1
            for (uint32_t t = 0; t < a.n; t++) {
                store_fe(SCR(t, 0), CHAIN_ROW, fe_mulv(Y, run));
                store_fe(SCR(t, 1), CHAIN_ROW, Z);
                run = fe_mulv(run, Z);
                add_cached(X, Y, Z, T, words_fe(a.step_ypx), words_fe(a.step_ymx), words_fe(a.step_t2d));
            }
            if (L > 1) add_cached(X, Y, Z, T, words_fe(a.jump_ypx), words_fe(a.jump_ymx), words_fe(a.jump_t2d));
            fe acc = block_invert(run);  // one inversion for the block's lanes
            const uint32_t base_step = r * a.n;
#pragma unroll 1
            for (uint32_t t = a.n; t-- > 0;) {
                const fe v = fe_mulv(load_fe(SCR(t, 0), CHAIN_ROW), acc);
                acc = fe_mulv(acc, load_fe(SCR(t, 1), CHAIN_ROW));
                test_emit(sink, v, lane, base_step + t);
            }
        }
        store_fe(a.lanes + 0 * L + lane, L, X);
        store_fe(a.lanes + 2 * L + lane, L, Y);
        store_fe(a.lanes + 4 * L + lane, L, Z);
        store_fe(a.lanes + 6 * L + lane, L, T);
    }
#undef SCR
}

// The filter a suffix-bitmap survivor matches (suffix_match), with the
// survivor's scalar offset over 8 decoded from its record.
__device__ __noinline__ uint32_t suffix_owner(const MatchArgs& a, const HitRec& r) {
    const uint64_t w = a.window0 + (uint64_t)(r.step / a.slots) * a.lanes + r.lane;
    const uint64_t k = w * a.slots + (a.paired ? 1u : 0u) + r.step % a.slots;
    const SuffixTables t{a.suffixes, a.nsuffix, a.pow8};
    bool bad = false;
    const uint32_t j = suffix_match(t, a.sx, a.sy, a.sz, a.st, k, r.y, bad);
    if (bad) atomicAdd(a.mismatch, 1u);
    return j == 0xffffffffu ? j : a.prefix_count + j;
}

// Exact match of one advance's bitmap survivors (grid-stride; the survivor
// count is read on the device, so the launch needs no host round trip).
__global__ void __launch_bounds__(128) match_kernel(const MatchArgs a) {
    const uint32_t n = min(*a.surv_count, a.surv_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const HitRec r = a.surv[i];
        uint32_t owner = (a.t.nbuckets || a.t.npatterns) ? exact_owner(a.t, r.y) : 0xffffffffu;
        if (owner == 0xffffffffu && a.sbitmap) {
            fe y;
#pragma unroll
            for (int q = 0; q < 8; q++) y.v[q] = r.y[q];
            const uint32_t slot = suffix_slot(y, a.sbits);
            if ((__ldg(a.sbitmap + (slot >> 5)) >> (slot & 31)) & 1u) owner = suffix_owner(a, r);
        }
        if (owner != 0xffffffffu) {
            const uint32_t idx = atomicAdd(a.out_count, 1u);
            if (idx < a.out_cap) {
                // window w = window0 + round * lanes + lane; candidate i of it
                const uint64_t w = a.window0 + (uint64_t)(r.step / a.slots) * a.lanes + r.lane;
                const uint64_t k = w * a.slots + (a.paired ? 1u : 0u) + r.step % a.slots;
                uint4* dst = reinterpret_cast<uint4*>(a.out + idx);
                dst[0] = make_uint4((uint32_t)(8 * k), (uint32_t)((8 * k) >> 32), r.y[0], r.y[1]);
                dst[1] = make_uint4(r.y[2], r.y[3], r.y[4], r.y[5]);
                dst[2] = make_uint4(r.y[6], r.y[7], owner, 0u);
            }
        }
    }
}

}  // namespace

cudaError_t launch_match(const MatchArgs& a, int grid, cudaStream_t s) {
    match_kernel<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_init(const InitArgs& a, int block, cudaStream_t s) {
    const unsigned grid = (a.lanes_n + block - 1) / block;
    init_kernel<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_paired(const PairedArgs& a, int block, int grid, cudaStream_t s) {
    const uint32_t n = a.lanes_per_thread;
    if ((n != 1 && n != 2) || block % 32 != 0 || grid <= 0 || a.lanes_n % ((uint32_t)block * n) != 0 ||
        a.slots_n != (uint32_t)grid * (uint32_t)block * n)
        return cudaErrorInvalidValue;
    if (n == 2)
        paired_kernel2<<<grid, block, 0, s>>>(a);
    else if (a.stage_records)
        paired_kernel<true><<<grid, block, 0, s>>>(a);
    else
        paired_kernel<false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_chain(const ChainArgs& a, int block, int grid, cudaStream_t s) {
    if (a.lanes_n % block != 0 || block % 32 != 0 || grid < 1 || (uint32_t)grid * block != a.slots_n)
        return cudaErrorInvalidValue;
    const size_t smem = (a.bitmap && a.bits <= STAGED_BITMAP_BITS) ? (size_t)(1u << a.bits) / 8u : 0;
    chain_kernel<<<grid, block, smem, s>>>(a);
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

cudaError_t paired_info(int block, uint32_t, uint32_t lanes_per_thread, KernelInfo* info) {
    return info_of(lanes_per_thread == 2 ? (const void*)paired_kernel2 : (const void*)paired_kernel<true>, block, 0, info);
}

// sized for a staged 16-bit bitmap, the most a chain launch takes
cudaError_t chain_info(int block, KernelInfo* info) {
    return info_of((const void*)chain_kernel, block, (size_t)(1u << STAGED_BITMAP_BITS) / 8u, info);
}

}  // namespace og
