// og_search_noalloc: the paired search without any device allocation.
//
// Some callers cannot allocate device memory: code running inside another
// framework's memory pool that forbids cudaMalloc behind its back, callers
// that must not synchronise the device (cudaMalloc and cudaFree can), and
// processes that reserve all device memory up front. This entry point lets
// them run the search: they pass the inputs (start point, bitmap) and the
// outputs (survivor records and their counter) in device memory they own,
// and everything else — lane state, the Montgomery scratch and the tables —
// lives in one file-scope device array, `og_noalloc_scratch`, sized
// OG_NOALLOC_SCRATCH_BYTES. Every GPU that loads the library holds that array
// until the process exits.
//
// Host code must not use the array's name as a device address (in host code
// it is a host-side stand-in); it takes the address once per device with
// cudaGetSymbolAddress, on the first call made on that device, and passes it
// to the kernels.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/onion_gen_b200.h"
#include "host/common.h"
#include "search_common.cuh"

namespace og {
namespace {

constexpr size_t SCRATCH_BYTES = OG_NOALLOC_SCRATCH_BYTES;
constexpr uint32_t NBLOCK = 128;
static_assert(NBLOCK <= PARK_STRIDE, "paired_rounds parks PARK_STRIDE lanes per block");
constexpr uint32_t POW2 = 24;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) uint4 og_noalloc_scratch[SCRATCH_BYTES / sizeof(uint4)];

// Layout inside the array, in uint4 units: the table Q_m (half * 6), the
// lane centres (lanes * 4) and the Montgomery scratch
// (lanes * (2 half + 2) * 4).
size_t need_uint4(uint32_t lanes, uint32_t half) {
    return (size_t)half * 6 + (size_t)lanes * 4 + (size_t)lanes * (2 * (size_t)half + 2) * 4;
}

// 2^k p for k < POW2 in cached form (y + x, y - x, 2 d x y; Z = 1), passed to
// the kernels by value as a launch parameter (2304 bytes), so that the call
// copies nothing from host memory: a host-to-device copy from pageable
// memory would wait for the work already queued on the caller's stream.
struct Pow2Table {
    uint4 v[POW2 * 6];
};

struct NoAllocArgs {
    uint4* table;
    uint4* lanes;
    uint4* scratch;
    FeWords bx, by, bz, bt;  // first centre, extended
    FeWords ex, ey, ez, et;  // 8G, extended (table entry 1)
    FeWords wx, wy, wt;      // round stride, affine
    const uint32_t* bitmap;
    uint32_t bits;
    HitRec* hits;
    uint32_t* counter;
    uint32_t cap;
    uint32_t lanes_n;
    uint32_t half;
    uint32_t rounds;
};

// The table Q_m = m * 8G, m = 1..half, affine with x y. Entry m - 1 starts
// from 8G and adds 2^k * 8G (from `pow8`) for every bit k of m - 1, then is
// normalised.
__global__ void __launch_bounds__(NBLOCK) noalloc_table_kernel(const NoAllocArgs a, const Pow2Table pow8) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.half) return;
    fe X = words_fe(a.ex), Y = words_fe(a.ey), Z = words_fe(a.ez), T = words_fe(a.et);
    for (uint32_t k = 0; k < POW2; k++)
        if ((m >> k) & 1u) {
            const uint4* p = pow8.v + (size_t)k * 6;
            add_cached(X, Y, Z, T, load_fe(p + 0, 1), load_fe(p + 2, 1), load_fe(p + 4, 1));
        }
    const fe zi = fe_invert(Z);
    const fe x = fe_mulv(X, zi), y = fe_mulv(Y, zi);
    uint4* d = a.table + (size_t)m * 6;
    store_fe(d + 0, 1, x);
    store_fe(d + 2, 1, y);
    store_fe(d + 4, 1, fe_mulv(x, y));
}

// Lane l starts on the centre of window l: the first centre plus 2^k times
// the lane stride (from `pow2`) for every bit k of l.
__global__ void __launch_bounds__(NBLOCK) noalloc_init_kernel(const NoAllocArgs a, const Pow2Table pow2) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= a.lanes_n) return;
    const size_t L = a.lanes_n;
    fe X = words_fe(a.bx), Y = words_fe(a.by), Z = words_fe(a.bz), T = words_fe(a.bt);
    for (uint32_t k = 0; k < POW2; k++)
        if ((lane >> k) & 1u) {
            const uint4* p = pow2.v + (size_t)k * 6;
            add_cached(X, Y, Z, T, load_fe(p + 0, 1), load_fe(p + 2, 1), load_fe(p + 4, 1));
        }
    const fe zi = fe_invert(Z);
    store_fe(a.lanes + 0 * L + lane, L, fe_mulv(X, zi));
    store_fe(a.lanes + 2 * L + lane, L, fe_mulv(Y, zi));
}

// The production paired kernel with its scratch in the file-scope array; the
// table is read through L1 as in the single engine.
__global__ void __launch_bounds__(NBLOCK, 5) noalloc_paired_kernel(const NoAllocArgs a) {
    const uint4* qtab = a.table;
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t L = a.lanes_n;
    const Sink sink{a.bitmap, a.bits, a.hits, a.counter, a.cap, 0, nullptr, 0};
    fe x = load_fe(a.lanes + 0 * L + lane, L);
    fe y = load_fe(a.lanes + 2 * L + lane, L);
    paired_rounds<true>(x, y, words_fe(a.wx), words_fe(a.wy), words_fe(a.wt), qtab, a.half, a.rounds, a.scratch + lane, L,
                  [&](const fe& v, uint32_t step) { test_emit(sink, v, lane, step); });
}

// The array's device address, per device, taken on the first call there.
std::mutex g_mu;
uint4* g_addr[MAX_DEVICES];

// 2^k * p for k < POW2 in cached form.
void pow2_into(Pt p, uint4* out) {
    for (uint32_t k = 0; k < POW2; k++) {
        const Niels c = pt_niels(p);
        put_fe(out + k * 6 + 0, 1, c.ypx);
        put_fe(out + k * 6 + 2, 1, c.ymx);
        put_fe(out + k * 6 + 4, 1, c.xy2d);
        p = pt_dbl(p);
    }
}

}  // namespace
}  // namespace og

using namespace og;

extern "C" int og_search_noalloc(int ordinal, const uint8_t start[128], uint32_t lanes, uint32_t half, uint32_t rounds,
                                 const uint32_t* d_bitmap, uint32_t bits, og_hit_record* d_hits, uint32_t cap,
                                 uint32_t* d_count, void* stream, char* err, size_t errlen) {
    if (!start || !d_hits || !d_count) return fail(err, errlen, OG_E_ARG, "null argument");
    if (ordinal < 0 || ordinal >= MAX_DEVICES) return fail(err, errlen, OG_E_ARG, "device %d", ordinal);
    if (lanes == 0 || lanes % NBLOCK)
        return fail(err, errlen, OG_E_ARG, "lanes %u: a positive multiple of %u", lanes, NBLOCK);
    if (half == 0 || half > 2048) return fail(err, errlen, OG_E_ARG, "half %u outside 1..2048", half);
    if (rounds == 0) return fail(err, errlen, OG_E_ARG, "zero rounds");
    if ((uint64_t)rounds * (2ULL * half + 1) > 0xffffffffULL) return fail(err, errlen, OG_E_ARG, "too many rounds");
    if (d_bitmap && (bits < 8 || bits > 32)) return fail(err, errlen, OG_E_ARG, "bitmap width %u outside 8..32", bits);
    if (lanes >= (1u << POW2)) return fail(err, errlen, OG_E_ARG, "lanes %u", lanes);
    const size_t need = need_uint4(lanes, half) * sizeof(uint4);
    if (need > SCRATCH_BYTES)
        return fail(err, errlen, OG_E_CAPACITY,
                    "%u lanes at half %u need %zu bytes of scratch; the fixed array holds %zu "
                    "(lanes * (2 half + 3) * 64 + half * 96 must stay within it)",
                    lanes, half, need, SCRATCH_BYTES);
    const Pt A = point_from_bytes(start);
    if (!point_valid(A)) return fail(err, errlen, OG_E_ARG, "the start point is not on the curve");
    cudaError_t e = cudaSetDevice(ordinal);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "cudaSetDevice: %s", cuda_text(e).c_str());
    uint4* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[ordinal]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, og_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return fail(err, errlen, OG_E_DEVICE, "cudaGetSymbolAddress: %s", cuda_text(e).c_str());
            g_addr[ordinal] = static_cast<uint4*>(p);
        }
        base = g_addr[ordinal];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NoAllocArgs a;
    std::memset(&a, 0, sizeof a);
    a.table = base;
    a.lanes = a.table + (size_t)half * 6;
    a.scratch = a.lanes + (size_t)lanes * 4;
    const uint32_t slots = 2 * half + 1;
    // constants computed on the host and passed as launch parameters: the
    // first centre, 8G, the round stride
    const Pt first = pt_add(A, base_mult_u64(8ULL * (half + 1)));
    a.bx = to_words(first.X);
    a.by = to_words(first.Y);
    a.bz = to_words(first.Z);
    a.bt = to_words(first.T);
    const Pt eight = base_mult_u64(8);
    a.ex = to_words(eight.X);
    a.ey = to_words(eight.Y);
    a.ez = to_words(eight.Z);
    a.et = to_words(eight.T);
    F51 wx, wy;
    pt_affine(base_mult_u64(8ULL * slots * lanes), wx, wy);
    a.wx = to_words(wx);
    a.wy = to_words(wy);
    a.wt = to_words(f_mul(wx, wy));
    a.bitmap = d_bitmap;
    a.bits = bits;
    a.hits = reinterpret_cast<HitRec*>(d_hits);
    a.counter = d_count;
    a.cap = cap;
    a.lanes_n = lanes;
    a.half = half;
    a.rounds = rounds;
    // the two power-of-two tables travel as launch parameters
    Pow2Table pow2, pow8;
    pow2_into(base_mult_u64(8ULL * slots), pow2.v);
    pow2_into(eight, pow8.v);
    // the counter starts at zero on every call
    e = cudaMemsetAsync(d_count, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "memset: %s", cuda_text(e).c_str());
    noalloc_table_kernel<<<(half + NBLOCK - 1) / NBLOCK, NBLOCK, 0, s>>>(a, pow8);
    noalloc_init_kernel<<<lanes / NBLOCK, NBLOCK, 0, s>>>(a, pow2);
    noalloc_paired_kernel<<<lanes / NBLOCK, NBLOCK, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "launch: %s", cuda_text(e).c_str());
    return OG_OK;
}
