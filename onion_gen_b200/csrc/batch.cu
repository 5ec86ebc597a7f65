// og_batch: many independent searches advancing together in one persistent
// kernel, replayed as a CUDA graph per step. No counterpart in the reference;
// the per-search arithmetic is the single engine's paired round.
//
// Candidate windows. A search runs at its own inversion batch `half`; its
// window w is the round centred on scalar offset 8 (w (2 half + 1) + half + 1),
// whose 2 half + 1 candidates are offsets 8 (w (2 half + 1) + 1 + i),
// i in [0, 2 half]. A search holding L lanes for a step of R rounds processes
// windows [W, W + R L) — lane l takes W + r L + l in round r — and ends the
// step with lane l centred on window W + R L + l. So after every step lane l
// sits on window W_done + l whatever L was: a search that grows only
// initialises its new lanes, one that shrinks drops its highest lanes, and
// the windows it has processed are always exactly [0, W_done).
//
// Results. A search is done when it holds `quota` verified hits; because its
// windows are processed in increasing order, these are its first `quota`
// hits in offset order, a pure function of the search alone (whatever its
// half, lanes or neighbours).
//
// Steps in flight. og_batch_step keeps up to `inflight` steps queued on the
// device (two by default): it launches the next step, then collects the
// oldest one (waits for it, copies its exact hits back on a stream of their
// own and re-derives them on the host) while the newer one runs. A step is
// planned from what the host knows when it launches it, so a search that
// meets its quota in the step still in flight keeps its lanes for one more
// step. The device does not run them: the exact-match kernel counts every
// search's exact hits, and the search kernel returns at once from a block of
// a search whose count has reached its quota. Per-search tables come from a
// stream-ordered pool and are freed in stream order, so admitting or
// retiring a search never waits for the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/onion_gen_b200.h"
#include "host/common.h"
#include "host/filters.h"
#include "host/keys.h"
#include "host/tuning.h"
#include "search_common.cuh"
#include "suffix_match.cuh"

#ifndef OG_LB_THREADS
#define OG_LB_THREADS 128
#endif
#ifndef OG_LB_MIN_BLOCKS
#define OG_LB_MIN_BLOCKS 5
#endif

namespace og {

const std::vector<uint4>& pair_table(uint32_t half);           // engine.cu
std::vector<uint4> pow2_table(const Pt& stride, uint32_t nbits);  // engine.cu
MatchTables match_tables(const std::vector<FilterSet::DeviceBucket>& buckets, const uint64_t* keys,
                         const uint32_t* owners, const uint32_t* patterns,
                         uint32_t npatterns);                      // engine.cu

namespace {

constexpr uint32_t BLOCK = 128;
constexpr uint32_t NONE = 0xffffffffu;
constexpr int MAX_BUCKETS = MAX_MATCH_BUCKETS;
constexpr uint32_t POW2_BITS = 24;  // lanes of one search stay below 2^24
constexpr uint32_t MAX_HALF = 2048;
constexpr int FLIGHTS = 2;
// A filter set whose bitmap lets more than this fraction of candidates
// through is refused: the survivor buffer is sized from it.
constexpr double MAX_OCCUPANCY = 0.02;
// With max_half above half, a search runs at a doubled half while its
// expected work covers at least this many steps of the whole pool there.
constexpr double LONG_STEPS = 4.0;
// A search needs the blocks that cover its expected remaining work in this
// many steps.
constexpr double NEED_STEPS = 2.0;
// shared memory of the search kernel: a staged bitmap of STAGED_BITMAP_BITS
constexpr size_t STAGED_BYTES = (size_t)(1u << STAGED_BITMAP_BITS) / 8u;

struct BatchDesc {
    FeWords wx, wy, wt;      // the search's stride for this step: L (2 half + 1) 8 G, affine
    FeWords bx, by, bz, bt;  // centre of window W_done (where new lanes start), extended
    const uint32_t* bitmap;  // prefix bitmap (nullptr: the search has no prefix)
    uint32_t bits;
    uint32_t half;           // the search's inversion batch: a round is 2 half + 1 candidates
    MatchTables match;
    const uint32_t* sbitmap;  // suffix bitmap (nullptr: no suffix)
    uint32_t sbits;
    uint32_t prefix_count;    // filter index of suffix j is prefix_count + j
    const uint32_t* suffixes; // the suffix patterns (SuffixTables layout)
    uint32_t nsuffix;
    uint32_t quota;           // exact hits after which the device skips the search's blocks (0: never)
    const uint4* pow2;        // 2^k (2 half + 1) 8 G, k < POW2_BITS, cached: new lanes' start points
    FeWords sx, sy, sz, st;   // the search's start point s B, extended
};

// Where a search stands in a step: the windows done before it and the
// lanes it runs (a survivor's offset is decoded from them on the device).
struct SearchPos {
    uint64_t windows;
    uint32_t lanes;
    uint32_t pad;
};

struct SlotBlock {
    uint32_t sidx;   // descriptor index, NONE when the block is idle
    uint32_t lane0;  // lane index (within its search) of the block's first slot
};

struct Counters {
    uint32_t work;        // next work item of the persistent kernel
    uint32_t init_count;  // slot blocks in the init list
    uint32_t surv;        // bitmap survivors written
    uint32_t hits;        // exact hits written
    uint32_t mismatch;    // suffix survivors whose recomputed key differed
    uint32_t pad[3];
};

struct BatchArgs {
    const BatchDesc* descs;
    const SlotBlock* blocks;
    const uint32_t* init_list;
    Counters* counters;  // the flight's
    uint32_t nblocks;
    uint4* lanes;    // ({x,y} * 2 + q) * slots + slot
    // per persistent CTA, a region of cta_scratch uint4 in which thread t's
    // element e, part w, half q is at ((e * 2 + w) * 2 + q) * BLOCK + t
    uint4* scratch;
    size_t cta_scratch;
    size_t slots;
    const uint4* table;  // Q_m, m = 1..max half; a search of half h reads the first h
    uint32_t rounds;
    HitRec* surv;  // the flight's
    uint32_t surv_cap;
    HitRec* hits;  // the flight's
    uint32_t hit_cap;
    const SearchPos* pos;  // per descriptor
    const uint4* pow8;     // 2^j 8G, j < 64, for the suffix key recomputation
    uint32_t* found;       // per descriptor: exact hits counted on the device so far
    uint32_t* mism;        // per descriptor: suffix survivors whose recomputed key differed
};

__global__ void __launch_bounds__(BLOCK) batch_init_kernel(const BatchArgs a) {
    if (blockIdx.x >= a.counters->init_count) return;
    const uint32_t b = a.init_list[blockIdx.x];
    const SlotBlock sb = a.blocks[b];
    const BatchDesc& d = a.descs[sb.sidx];
    const uint32_t lane = sb.lane0 + threadIdx.x;
    const size_t slot = (size_t)b * BLOCK + threadIdx.x;
    fe X = words_fe(d.bx), Y = words_fe(d.by), Z = words_fe(d.bz), T = words_fe(d.bt);
    for (uint32_t k = 0; k < POW2_BITS; k++) {
        if ((lane >> k) & 1u) {
            const uint4* p = d.pow2 + (size_t)k * 6;
            add_cached(X, Y, Z, T, load_fe(p + 0, 1), load_fe(p + 2, 1), load_fe(p + 4, 1));
        }
    }
    const fe zi = fe_invert(Z);
    store_fe(a.lanes + 0 * a.slots + slot, a.slots, fe_mulv(X, zi));
    store_fe(a.lanes + 2 * a.slots + slot, a.slots, fe_mulv(Y, zi));
}

// Persistent: one CTA per resident slot, each pulling slot blocks until the
// pool is exhausted. Every block of lanes belongs to one search, whose
// descriptor gives its half, stride and bitmap. A block of a search whose
// exact hits have reached its quota (counted by the previous steps' exact
// kernels) is skipped: its lanes stay where they are. A prefix bitmap of up
// to 16 bits is staged in shared memory, again only when the CTA's next
// block belongs to another search (config 4 on B200: 19.52-19.55 s against
// 19.67-19.82 s, the searches' small bitmaps no longer competing with the
// table Q_m for L1).
__global__ void __launch_bounds__(OG_LB_THREADS, OG_LB_MIN_BLOCKS) batch_search_kernel(const BatchArgs a) {
    const uint4* qtab = a.table;  // read through L1, as the single-search kernel does
    __shared__ uint32_t item_s, staged_s;  // staged_s: the search whose bitmap is in og_bitmap_s
    if (threadIdx.x == 0) staged_s = NONE;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_s = atomicAdd(&a.counters->work, 1u);
        __syncthreads();
        const uint32_t item = item_s;
        if (item >= a.nblocks) break;
        const SlotBlock sb = a.blocks[item];
        if (sb.sidx == NONE) continue;
        const BatchDesc& d = a.descs[sb.sidx];
        if (d.quota && a.found[sb.sidx] >= d.quota) continue;
        // the block's search decides this, the same for every thread; the
        // barrier at the loop's top has retired every read of the old map
        const bool staged = d.bitmap && d.bits <= STAGED_BITMAP_BITS;
        if (staged && staged_s != sb.sidx) {
            extern __shared__ uint32_t og_bitmap_s[];
            const uint32_t words = (1u << d.bits) / 32u;
            for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) og_bitmap_s[i] = d.bitmap[i];
            __syncthreads();
            if (threadIdx.x == 0) staged_s = sb.sidx;
        }
        const uint32_t slot = item * BLOCK + threadIdx.x;
        const Sink sink{d.bitmap, d.bits, a.surv, &a.counters->surv, a.surv_cap, sb.sidx, d.sbitmap, d.sbits, staged};
        fe x = load_fe(a.lanes + 0 * a.slots + slot, a.slots);
        fe y = load_fe(a.lanes + 2 * a.slots + slot, a.slots);
        paired_rounds<false>(x, y, words_fe(d.wx), words_fe(d.wy), words_fe(d.wt), qtab, d.half, a.rounds,
                      a.scratch + blockIdx.x * a.cta_scratch + threadIdx.x, (size_t)BLOCK,
                      [&](const fe& v, uint32_t step) { test_emit(sink, v, slot, step); });
        store_fe(a.lanes + 0 * a.slots + slot, a.slots, x);
        store_fe(a.lanes + 2 * a.slots + slot, a.slots, y);
    }
}

// Exact match of the bitmap survivors: per distinct filter length, a binary
// search of the sorted masked key heads (FilterSet::match_key on the device);
// every exact hit is counted for its search.
__global__ void __launch_bounds__(256) batch_exact_kernel(const BatchArgs a) {
    const uint32_t n = min(a.counters->surv, a.surv_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const HitRec r = a.surv[i];
        const BatchDesc& d = a.descs[r.search];
        uint32_t owner = (d.match.nbuckets || d.match.npatterns) ? exact_owner(d.match, r.y) : NONE;
        if (owner == NONE && d.sbitmap) {
            fe y;
#pragma unroll
            for (int q = 0; q < 8; q++) y.v[q] = r.y[q];
            const uint32_t slot = suffix_slot(y, d.sbits);
            if ((__ldg(d.sbitmap + (slot >> 5)) >> (slot & 31)) & 1u) {
                // lane l of the search at round r of this step covers window
                // W_done + r L + l; its candidate i has scalar offset
                // 8 (w (2 half + 1) + 1 + i)
                const SearchPos p = a.pos[r.search];
                const uint32_t slots = 2 * d.half + 1;
                const uint64_t lane = a.blocks[r.lane / BLOCK].lane0 + r.lane % BLOCK;
                const uint64_t w = p.windows + (uint64_t)(r.step / slots) * p.lanes + lane;
                const uint64_t k = w * slots + 1 + r.step % slots;
                const SuffixTables t{d.suffixes, d.nsuffix, a.pow8};
                bool bad = false;
                const uint32_t j = suffix_match(t, d.sx, d.sy, d.sz, d.st, k, r.y, bad);
                if (bad) {
                    atomicAdd(&a.counters->mismatch, 1u);
                    atomicAdd(a.mism + r.search, 1u);
                }
                if (j != NONE) owner = d.prefix_count + j;
            }
        }
        if (owner != NONE) {
            atomicAdd(a.found + r.search, 1u);
            const uint32_t idx = atomicAdd(&a.counters->hits, 1u);
            if (idx < a.hit_cap) {
                HitRec h = r;
                h.pad = owner;
                a.hits[idx] = h;
            }
        }
    }
}

// The tuning.yaml key of the batch's shape on a device.
std::string batch_key(int ordinal) {
    char name[256] = "unnamed";
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, ordinal) == cudaSuccess) snprintf(name, sizeof name, "%s", p.name);
    return device_key(name, "cuda-batch", 0);
}

// A device allocation from the batch's stream-ordered pool: allocated on the
// upload stream, freed in the order of the engine's stream, so that a step
// still in flight keeps reading it until it ends.
template <typename T>
struct PoolBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t free_on = nullptr;
    PoolBuf() = default;
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    ~PoolBuf() { reset(); }
    cudaError_t alloc(size_t count, cudaMemPool_t pool, cudaStream_t on, cudaStream_t free_stream) {
        reset();
        if (count == 0) return cudaSuccess;
        void* q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, count * sizeof(T), pool, on);
        if (e != cudaSuccess) return e;
        p = static_cast<T*>(q);
        n = count;
        free_on = free_stream;
        return cudaSuccess;
    }
    void reset() {
        if (p) cudaFreeAsync(p, free_on);
        p = nullptr;
        n = 0;
    }
};

struct Search {
    uint64_t id = 0;
    uint8_t seed[32];
    uint8_t scalar[32];
    Pt start;
    FilterSet fs;
    SuffixSet sfx;
    bool has_prefixes = false;
    bool has_suffixes = false;
    bool long_filters = false;  // some hit needs the host's confirmation beyond the device match
    uint32_t quota = 0;
    uint32_t half = 0;
    double prob = 0;  // chance that a candidate matches one of its filters
    uint32_t sidx = NONE;
    PoolBuf<uint32_t> bitmap;
    PoolBuf<uint64_t> keys;
    PoolBuf<uint32_t> owners;
    PoolBuf<uint32_t> sbitmap, suffixes, patterns;
    std::vector<FilterSet::DeviceBucket> buckets;
    uint64_t table_bytes = 0;
    uint64_t windows = 0;            // windows of the steps launched so far
    uint64_t windows_collected = 0;  // windows of the steps collected: processed
    std::vector<uint32_t> blocks;    // slot blocks held, in lane order
    uint32_t lanes_last = 0;         // lanes held in the last step launched
    uint32_t lanes_stride = 0;       // lane count the descriptor's stride is for
    std::vector<og_batch_hit> hits;  // verified, in offset order
    bool done = false;
    uint32_t status = OG_OK;         // OG_E_VERIFY when a device hit did not re-derive
    uint64_t admit_order = 0;
};

// The searches a launched step runs, as planned at its launch.
struct Planned {
    uint64_t id;
    uint64_t admit_order;  // tells the search apart from a later one admitted under the same id
    uint32_t sidx;
    uint32_t half;
    uint32_t lanes;
    bool skippable;     // the device skips it once its quota is counted
    uint64_t windows0;  // its W_done when the step starts
};

// One step's buffers: what the device writes while a newer step may already
// be running, and the host staging of what the step's launch uploaded.
struct Flight {
    DevBuf<Counters> counters;
    DevBuf<HitRec> surv, hits;
    HostBuf<Counters> h_counters;
    HostBuf<BatchDesc> h_descs;   // descriptors uploaded at this launch
    HostBuf<SlotBlock> h_blocks;  // the block table this step ran (decodes its records)
    HostBuf<uint32_t> h_init;     // init list, then its length at [nblocks]
    HostBuf<SearchPos> h_pos;
    BatchArgs args{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool pending = false;
    std::vector<Planned> plan;

    ~Flight() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

}  // namespace
}  // namespace og

using namespace og;

struct og_batch {
    int device = 0;
    cudaStream_t stream = nullptr;   // the steps
    cudaStream_t ustream = nullptr;  // uploads of admitted searches' tables
    cudaStream_t cstream = nullptr;  // a collected step's hits, while the next step runs
    cudaMemPool_t pool = nullptr;
    og_batch_config cfg{};
    uint32_t slots = 0, nblocks = 0, grid = 0;
    DevBuf<uint4> lanes, scratch, table, pow8;
    std::map<uint32_t, DevBuf<uint4>> pow2;  // per half
    DevBuf<BatchDesc> descs;
    DevBuf<SearchPos> pos;
    DevBuf<SlotBlock> blocks;
    DevBuf<uint32_t> init_list;
    DevBuf<uint32_t> found, mism;
    std::vector<BatchDesc> h_descs;     // the descriptors as the host has them
    std::vector<SlotBlock> h_blocks;    // the block table as the host has it
    HostBuf<HitRec> h_hits;
    HostBuf<uint32_t> h_mism;
    Flight flights[FLIGHTS];
    uint64_t launched = 0, collected = 0;
    uint32_t suffix_searches = 0;  // admitted searches with suffixes
    std::map<uint64_t, std::unique_ptr<Search>> searches;
    std::vector<uint32_t> free_sidx;
    std::vector<uint32_t> free_blocks;
    std::map<std::pair<uint32_t, uint32_t>, std::array<FeWords, 3>> strides;  // per (lanes, half)
    uint64_t admitted = 0;
    uint64_t mem_used = 0, mem_budget = 0;
    bool active_changed = true;
    bool closed = false;
    std::string closed_why;
    float last_ms = 0;
    uint64_t last_candidates = 0;
    uint32_t last_launches = 0;
    uint32_t dirty_lo = NONE, dirty_hi = 0;
    std::set<uint64_t> planted;  // searches whose next hit is treated as not re-deriving (tests)

    ~og_batch() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (ustream) cudaStreamSynchronize(ustream);
        searches.clear();  // their tables go back to the pool in stream order
        if (stream) cudaStreamSynchronize(stream);
        if (stream) cudaStreamDestroy(stream);
        if (ustream) cudaStreamDestroy(ustream);
        if (cstream) cudaStreamDestroy(cstream);
        if (pool) cudaMemPoolDestroy(pool);
    }

    void mark(uint32_t sidx) {
        dirty_lo = std::min(dirty_lo, sidx);
        dirty_hi = std::max(dirty_hi, sidx + 1);
    }

    uint32_t pending() const { return (uint32_t)(launched - collected); }
};

namespace {

#define CU(call)                                                                                 \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess)                                                                   \
            return fail(err, errlen, _e == cudaErrorMemoryAllocation ? OG_E_NOMEM : OG_E_DEVICE, \
                        "%s: %s", #call, cuda_text(_e).c_str());                                 \
    } while (0)

const std::array<FeWords, 3>& stride_for(og_batch* b, uint32_t lanes, uint32_t half) {
    const auto key = std::make_pair(lanes, half);
    auto it = b->strides.find(key);
    if (it != b->strides.end()) return it->second;
    F51 x, y;
    pt_affine(base_mult_u64(8ULL * (2ULL * half + 1) * lanes), x, y);
    std::array<FeWords, 3> w{to_words(x), to_words(y), to_words(f_mul(x, y))};
    return b->strides.emplace(key, w).first->second;
}

// Window W's centre for search s: s * B + 8 (W (2 half + 1) + half + 1) B.
Pt window_centre(const Search& s, uint64_t w) {
    const uint64_t k = 8ULL * (w * (2ULL * s.half + 1) + s.half + 1);
    return pt_add(s.start, base_mult_u64(k));
}

void release_blocks(og_batch* b, Search& s) {
    for (uint32_t blk : s.blocks) b->free_blocks.push_back(blk);
    s.blocks.clear();
}

// A search ends: done with its quota, or failed with `status`. Its lanes go
// back to the pool at the next launch.
void finish(og_batch* b, Search& s, uint32_t status) {
    s.done = true;
    s.status = status;
    release_blocks(b, s);
    b->active_changed = true;
}

// Shares the slot pool among unfinished searches by max-min fairness on
// their needs: a search needs the blocks that cover its expected remaining
// work ((quota - hits) over its match probability) in NEED_STEPS steps, at
// least one. In ascending need (then admission order), each search gets its
// need or an equal share of the blocks still unassigned, whichever is
// smaller: short searches get all they can use and finish within a few
// steps, long ones split the rest equally, and when there are more searches
// than blocks the longest wait. Blocks nobody needs are spread evenly.
// Searches well above their share drop their highest blocks; those below
// take free blocks, whose lanes are queued for initialisation. Which lanes
// a search holds never changes its results.
void rebalance(og_batch* b, std::vector<uint32_t>& init) {
    std::vector<Search*> running;
    for (auto& kv : b->searches)
        if (!kv.second->done) running.push_back(kv.second.get());
    std::vector<double> need(running.size());
    for (size_t i = 0; i < running.size(); i++) {
        const Search& s = *running[i];
        const double left = (double)(s.quota - std::min<size_t>(s.quota, s.hits.size()));
        const double work = s.prob > 0 ? left / s.prob : INFINITY;
        const double per_block = NEED_STEPS * (2.0 * s.half + 1) * b->cfg.rounds * BLOCK;
        need[i] = std::max(1.0, std::ceil(work / per_block));
    }
    std::vector<size_t> order(running.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        if (need[x] != need[y]) return need[x] < need[y];
        return running[x]->admit_order < running[y]->admit_order;
    });
    {
        std::vector<Search*> sorted(running.size());
        std::vector<double> sneed(running.size());
        for (size_t i = 0; i < order.size(); i++) {
            sorted[i] = running[order[i]];
            sneed[i] = need[order[i]];
        }
        running.swap(sorted);
        need.swap(sneed);
    }
    std::vector<uint32_t> target(running.size(), 0);
    uint32_t left = b->nblocks;
    for (size_t i = 0; i < running.size() && left; i++) {
        const uint32_t share = left / (uint32_t)(running.size() - i);
        target[i] = (uint32_t)std::min<double>(need[i], (double)share);
        left -= target[i];
    }
    // blocks beyond every need: evenly over the searches that hold some
    size_t held = 0;
    for (uint32_t t : target) held += t ? 1 : 0;
    for (size_t i = 0; i < running.size() && left && held; i++) {
        if (!target[i]) continue;
        const uint32_t extra = left / (uint32_t)held--;
        target[i] += extra;
        left -= extra;
    }
    // Shrink only searches well above their share (a quarter over, at least
    // one block), so that arrivals and departures do not reshuffle every
    // search by a block each time; the free blocks go to those below it.
    // While a search with a share holds no block at all, every search
    // shrinks to its share exactly, so that a new arrival never waits for a
    // departure.
    bool starving = false;
    for (size_t i = 0; i < running.size(); i++) starving |= target[i] > 0 && running[i]->blocks.empty();
    for (size_t i = 0; i < running.size(); i++) {
        Search& s = *running[i];
        const size_t slack = target[i] && !starving ? std::max<size_t>(1, target[i] / 4) : 0;
        if (s.blocks.size() <= target[i] + slack) continue;
        while (s.blocks.size() > target[i]) {
            b->free_blocks.push_back(s.blocks.back());
            s.blocks.pop_back();
        }
    }
    for (size_t i = 0; i < running.size(); i++) {
        Search& s = *running[i];
        const size_t had = s.blocks.size();
        while (s.blocks.size() < target[i] && !b->free_blocks.empty()) {
            s.blocks.push_back(b->free_blocks.back());
            b->free_blocks.pop_back();
        }
        if (s.blocks.size() > had) {
            // the new lanes start on windows W_done + lane, W_done counting
            // the steps already launched
            const Pt c = window_centre(s, s.windows);
            BatchDesc& d = b->h_descs[s.sidx];
            d.bx = to_words(c.X);
            d.by = to_words(c.Y);
            d.bz = to_words(c.Z);
            d.bt = to_words(c.T);
            b->mark(s.sidx);
            for (size_t j = had; j < s.blocks.size(); j++) init.push_back(s.blocks[j]);
        }
    }
    for (uint32_t i = 0; i < b->nblocks; i++) b->h_blocks[i] = SlotBlock{NONE, 0};
    for (Search* s : running)
        for (size_t j = 0; j < s->blocks.size(); j++) b->h_blocks[s->blocks[j]] = SlotBlock{s->sidx, (uint32_t)(j * BLOCK)};
}

int enqueue_step(og_batch* b, const BatchArgs& a, char* err, size_t errlen) {
    CU(cudaMemsetAsync(a.counters, 0, offsetof(Counters, init_count), b->stream));
    CU(cudaMemsetAsync(&a.counters->surv, 0, 3 * sizeof(uint32_t), b->stream));  // surv, hits, mismatch
    batch_init_kernel<<<b->nblocks, BLOCK, 0, b->stream>>>(a);
    CU(cudaGetLastError());
    batch_search_kernel<<<b->grid, BLOCK, STAGED_BYTES, b->stream>>>(a);
    CU(cudaGetLastError());
    batch_exact_kernel<<<b->grid, 256, 0, b->stream>>>(a);
    CU(cudaGetLastError());
    return OG_OK;
}

// Marks the batch unusable after an error that leaves its results in doubt;
// later calls fail with OG_E_STATE.
int close_batch(og_batch* b, int rc, const char* err) {
    b->closed = true;
    b->closed_why = err ? err : "an earlier error";
    return rc;
}

// Expected candidates until the quota: quota over the chance that a
// candidate matches one of the search's filters (the reference's estimate,
// src/estimate.rs:69-78, divides the same way).
double expected_work(const Search& s) {
    std::vector<double> suffixes;
    for (size_t j = 0; j < s.sfx.size(); j++) suffixes.push_back(s.sfx.pattern(j).probability());
    const double p = either_of({s.has_prefixes ? s.fs.match_probability() : 0.0, either_of(suffixes)});
    return p > 0 ? (double)s.quota / p : INFINITY;
}

// The search's inversion batch: the batch's half, doubled (up to max_half)
// while the search's expected work covers LONG_STEPS steps of the whole pool
// at the doubled half. Results do not depend on it.
uint32_t choose_half(const og_batch* b, const Search& s) {
    uint32_t h = b->cfg.half;
    const double work = expected_work(s);
    while (2 * h <= b->cfg.max_half && work >= LONG_STEPS * (2.0 * (2 * h) + 1) * b->slots * b->cfg.rounds) h *= 2;
    return h;
}

// Plans and launches one step on the next free flight; `launched` says
// whether anything ran (nothing does when no search holds lanes).
int launch(og_batch* b, bool& launched, char* err, size_t errlen) {
    launched = false;
    Flight& f = b->flights[b->launched % FLIGHTS];
    if (f.pending) return fail(err, errlen, OG_E_STATE, "no free step buffers");
    std::vector<uint32_t> init;
    if (b->active_changed) {
        rebalance(b, init);
        b->active_changed = false;
    }
    f.plan.clear();
    for (auto& kv : b->searches) {
        Search& s = *kv.second;
        if (s.done || s.blocks.empty()) continue;
        const uint32_t lanes = (uint32_t)s.blocks.size() * BLOCK;
        if (lanes != s.lanes_stride) {
            const auto& w = stride_for(b, lanes, s.half);
            BatchDesc& d = b->h_descs[s.sidx];
            d.wx = w[0];
            d.wy = w[1];
            d.wt = w[2];
            s.lanes_stride = lanes;
            b->mark(s.sidx);
        }
        f.plan.push_back(Planned{s.id, s.admit_order, s.sidx, s.half, lanes, b->h_descs[s.sidx].quota != 0, s.windows});
    }
    if (f.plan.empty()) return OG_OK;
    if (b->dirty_lo < b->dirty_hi) {
        const size_t lo = b->dirty_lo, m = b->dirty_hi - b->dirty_lo;
        std::memcpy(f.h_descs.p, b->h_descs.data() + lo, m * sizeof(BatchDesc));
        CU(cudaMemcpyAsync(b->descs.p + lo, f.h_descs.p, m * sizeof(BatchDesc), cudaMemcpyHostToDevice, b->stream));
        b->dirty_lo = NONE;
        b->dirty_hi = 0;
    }
    std::memcpy(f.h_blocks.p, b->h_blocks.data(), b->nblocks * sizeof(SlotBlock));
    CU(cudaMemcpyAsync(b->blocks.p, f.h_blocks.p, b->nblocks * sizeof(SlotBlock), cudaMemcpyHostToDevice, b->stream));
    if (b->suffix_searches) {
        // where each search stands, for the device's offset decode of its
        // suffix survivors
        uint32_t top = 0;
        for (const Planned& p : f.plan) {
            f.h_pos.p[p.sidx] = SearchPos{p.windows0, p.lanes, 0};
            top = std::max(top, p.sidx + 1);
        }
        CU(cudaMemcpyAsync(b->pos.p, f.h_pos.p, top * sizeof(SearchPos), cudaMemcpyHostToDevice, b->stream));
    }
    for (size_t i = 0; i < init.size(); i++) f.h_init.p[i] = init[i];
    if (!init.empty())
        CU(cudaMemcpyAsync(b->init_list.p, f.h_init.p, init.size() * 4, cudaMemcpyHostToDevice, b->stream));
    f.h_init.p[b->nblocks] = (uint32_t)init.size();
    CU(cudaMemcpyAsync(&f.counters.p->init_count, &f.h_init.p[b->nblocks], 4, cudaMemcpyHostToDevice, b->stream));
    CU(cudaEventRecord(f.ev0, b->stream));
    if (f.exec) {
        CU(cudaGraphLaunch(f.exec, b->stream));
    } else {
        int rc = enqueue_step(b, f.args, err, errlen);
        if (rc != OG_OK) return rc;
        CU(cudaMemcpyAsync(f.h_counters.p, f.counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, b->stream));
    }
    CU(cudaEventRecord(f.ev1, b->stream));
    for (const Planned& p : f.plan) {
        Search& s = *b->searches[p.id];
        s.windows += (uint64_t)b->cfg.rounds * p.lanes;
        s.lanes_last = p.lanes;
    }
    f.pending = true;
    b->launched++;
    launched = true;
    return OG_OK;
}

// Waits for the oldest step in flight and takes its results: decodes every
// exact hit's offset from the step's own plan and block table, and verifies
// each search's hits in offset order up to its quota.
int collect(og_batch* b, og_batch_hit* out, size_t cap, size_t* n, char* err, size_t errlen) {
    Flight& f = b->flights[b->collected % FLIGHTS];
    CU(cudaEventSynchronize(f.ev1));
    f.pending = false;
    b->collected++;
    cudaEventElapsedTime(&b->last_ms, f.ev0, f.ev1);
    b->last_launches = 3;
    const Counters c = *f.h_counters.p;
    if (c.surv > f.args.surv_cap || c.hits > f.args.hit_cap)
        return fail(err, errlen, OG_E_OVERFLOW, "a step produced %u survivors (room %u) and %u hits (room %u)", c.surv,
                    f.args.surv_cap, c.hits, f.args.hit_cap);
    if (c.mismatch) {
        // which searches' suffix survivors did not recompute (counts so far)
        CU(cudaMemcpyAsync(b->h_mism.p, b->mism.p, b->cfg.max_searches * 4, cudaMemcpyDeviceToHost, b->cstream));
        CU(cudaStreamSynchronize(b->cstream));
    }
    // the exact hits, on the copy stream: the next step runs on the engine's
    std::vector<HitRec> recs(c.hits);
    const size_t chunk = b->h_hits.n;
    for (size_t off = 0; off < c.hits; off += chunk) {
        const size_t m = std::min<size_t>(chunk, c.hits - off);
        CU(cudaMemcpyAsync(b->h_hits.p, f.hits.p + off, m * sizeof(HitRec), cudaMemcpyDeviceToHost, b->cstream));
        CU(cudaStreamSynchronize(b->cstream));
        std::memcpy(recs.data() + off, b->h_hits.p, m * sizeof(HitRec));
    }
    std::unordered_map<uint32_t, size_t> by_sidx;
    for (size_t i = 0; i < f.plan.size(); i++) by_sidx[f.plan[i].sidx] = i;
    std::vector<std::vector<og_batch_hit>> found(f.plan.size());
    for (const HitRec& h : recs) {
        const SlotBlock sb = f.h_blocks.p[h.lane / BLOCK];
        if (sb.sidx != h.search) continue;
        auto it = by_sidx.find(sb.sidx);
        if (it == by_sidx.end()) continue;
        const Planned& p = f.plan[it->second];
        const uint64_t slots_per_window = 2ULL * p.half + 1;
        const uint64_t lane = sb.lane0 + h.lane % BLOCK;
        const uint64_t r = h.step / slots_per_window, i = h.step % slots_per_window;
        const uint64_t w = p.windows0 + r * p.lanes + lane;
        og_batch_hit o{};
        o.search_id = p.id;
        o.offset = 8 * (w * slots_per_window + 1 + i);
        for (int k = 0; k < 8; k++)
            for (int j = 0; j < 4; j++) o.packed[4 * k + j] = (uint8_t)(h.y[k] >> (8 * j));
        o.filter = h.pad;
        found[it->second].push_back(o);
    }
    size_t emitted = 0;
    uint64_t candidates = 0;
    uint32_t failed = 0;
    for (size_t pi = 0; pi < f.plan.size(); pi++) {
        const Planned& p = f.plan[pi];
        auto sit = b->searches.find(p.id);
        // retired since its launch (and perhaps its id admitted again)
        if (sit == b->searches.end() || sit->second->admit_order != p.admit_order) continue;
        Search& s = *sit->second;
        if (s.done) {
            // finished in an earlier step: the device skipped its blocks
            // when it could count its quota, otherwise it ran them
            if (!p.skippable) candidates += (uint64_t)b->cfg.rounds * p.lanes * (2ULL * p.half + 1);
            continue;
        }
        candidates += (uint64_t)b->cfg.rounds * p.lanes * (2ULL * p.half + 1);
        s.windows_collected = p.windows0 + (uint64_t)b->cfg.rounds * p.lanes;
        if (c.mismatch && b->h_mism.p[p.sidx]) {
            finish(b, s, OG_E_VERIFY);
            failed++;
            continue;
        }
        std::vector<og_batch_hit>& v = found[pi];
        std::sort(v.begin(), v.end(), [](const og_batch_hit& x, const og_batch_hit& y) { return x.offset < y.offset; });
        bool bad = false;
        for (og_batch_hit& h : v) {
            if (s.hits.size() >= s.quota) break;
            const uint32_t np = s.has_prefixes ? (uint32_t)s.fs.size() : 0;
            if (h.filter < np && s.long_filters) {
                const long fi = s.fs.match_key(h.packed);
                if (fi < 0) continue;
                h.filter = (uint32_t)fi;
            }
            uint8_t pk[32];
            if (check_hit_scalar(s.scalar, h.offset, h.packed, pk) != HitCheck::ok || b->planted.erase(s.id)) {
                bad = true;
                break;
            }
            std::memcpy(h.public_key, pk, 32);
            if (h.filter < np) {
                // filters longer than the key-only span are confirmed on the address
                const PrefixFilter& pf = s.fs.filter(h.filter);
                if (pf.needs_full_check() && !pf.matches_address(address(pk))) continue;
            } else {
                // a suffix is confirmed on the re-derived key's address
                uint8_t addr[35];
                address_bytes(pk, addr);
                if (s.sfx.match_address(addr) != (long)(h.filter - np)) {
                    bad = true;
                    break;
                }
            }
            s.hits.push_back(h);
            if (out && emitted < cap) out[emitted] = h;
            emitted++;
        }
        if (bad) {
            finish(b, s, OG_E_VERIFY);
            failed++;
        } else if (s.hits.size() >= s.quota) {
            finish(b, s, OG_OK);
        }
    }
    b->last_candidates = candidates;
    *n = out ? std::min(emitted, cap) : 0;
    if (failed)
        return fail(err, errlen, OG_E_VERIFY,
                    "%u searches ended with OG_E_VERIFY: a device hit did not re-derive on the host (see their status)",
                    failed);
    if (out && emitted > cap) return fail(err, errlen, OG_E_CAPACITY, "%zu hits and room for %zu", emitted, cap);
    return OG_OK;
}

}  // namespace

extern "C" {

int og_batch_new(int ordinal, const og_batch_config* cfgp, og_batch** out, char* err, size_t errlen) {
    if (!out) return fail(err, errlen, OG_E_ARG, "null argument");
    *out = nullptr;
    og_batch_config cfg{};
    if (cfgp) cfg = *cfgp;
    // the fields that need no device first
    if (cfg.half > MAX_HALF || cfg.max_half > MAX_HALF)
        return fail(err, errlen, OG_E_ARG, "half %u / max_half %u (at most %u)", cfg.half, cfg.max_half, MAX_HALF);
    if (cfg.graph > 2) return fail(err, errlen, OG_E_ARG, "graph mode %u", cfg.graph);
    if (cfg.inflight > FLIGHTS) return fail(err, errlen, OG_E_ARG, "inflight %u (1 or %d)", cfg.inflight, FLIGHTS);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(err, errlen, OG_E_NODEVICE, "no CUDA device is available");
    if (ordinal < 0 || ordinal >= count) return fail(err, errlen, OG_E_ARG, "device %d of %d", ordinal, count);
    if (cfg.half == 0 && cfg.slots == 0 && cfg.rounds == 0 && cfg.grid == 0) {
        // the shape og_batch_tune recorded for this device, if any
        Shape s;
        if (tuning_get(batch_key(ordinal), s) && s.first && s.second) {
            cfg.half = s.first;
            cfg.slots = s.second;
            cfg.grid = s.block;
            cfg.rounds = s.rounds;
        }
    }
    if (cfg.half == 0) cfg.half = 256;
    if (cfg.half > MAX_HALF) return fail(err, errlen, OG_E_ARG, "half %u > %u", cfg.half, MAX_HALF);
    if (cfg.max_half == 0) cfg.max_half = cfg.half;
    if (cfg.max_half < cfg.half || cfg.max_half > MAX_HALF)
        return fail(err, errlen, OG_E_ARG, "max_half %u outside half %u .. %u", cfg.max_half, cfg.half, MAX_HALF);
    {
        uint32_t h = cfg.half;
        while (h < cfg.max_half) h *= 2;
        if (h != cfg.max_half) return fail(err, errlen, OG_E_ARG, "max_half %u is not half %u times a power of two", cfg.max_half, cfg.half);
    }
    if (cfg.rounds == 0) cfg.rounds = 1;
    if (cfg.max_searches == 0) cfg.max_searches = 4096;
    if (cfg.graph > 2) return fail(err, errlen, OG_E_ARG, "graph mode %u", cfg.graph);
    if (cfg.inflight == 0) cfg.inflight = 2;
    if (cfg.inflight > FLIGHTS) return fail(err, errlen, OG_E_ARG, "inflight %u (1 or %d)", cfg.inflight, FLIGHTS);
    CU(cudaSetDevice(ordinal));
    std::unique_ptr<og_batch> b(new (std::nothrow) og_batch());
    if (!b) return fail(err, errlen, OG_E_NOMEM, "host memory");
    b->device = ordinal;
    int per_sm = 0, sms = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_search_kernel, BLOCK, STAGED_BYTES));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ordinal));
    const uint32_t fit = (uint32_t)std::max(1, per_sm);
    cfg.grid = cfg.grid == 0 ? fit : std::min(cfg.grid, fit);
    b->grid = cfg.grid * (uint32_t)sms;
    if (cfg.slots == 0) cfg.slots = 2 * b->grid * BLOCK;
    cfg.slots = (cfg.slots + BLOCK - 1) / BLOCK * BLOCK;
    b->slots = cfg.slots;
    b->nblocks = cfg.slots / BLOCK;
    const uint64_t per_step = (uint64_t)cfg.slots * (2ULL * cfg.max_half + 1) * cfg.rounds;
    // survivors per step: at most MAX_OCCUPANCY of the candidates pass, a
    // sum of independent draws; room for that mean plus eight standard
    // deviations, at least 2^20
    const double mean = MAX_OCCUPANCY * (double)per_step;
    const uint64_t surv_cap = std::max<uint64_t>(1ULL << 20, (uint64_t)(mean + 8.0 * std::sqrt(mean) + 4096.0));
    if (surv_cap > 0x7fffffffULL) return fail(err, errlen, OG_E_ARG, "a step of %llu candidates is too large", (unsigned long long)per_step);
    if (cfg.max_hits == 0) cfg.max_hits = (uint32_t)surv_cap;
    b->cfg = cfg;

    CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&b->ustream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&b->cstream, cudaStreamNonBlocking));
    {
        // per-search tables: a pool of the batch's own, which never makes an
        // allocation wait for a step by adding a dependency of its own
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ordinal;
        CU(cudaMemPoolCreate(&b->pool, &props));
        int no = 0;
        CU(cudaMemPoolSetAttribute(b->pool, cudaMemPoolReuseAllowInternalDependencies, &no));
    }
    const size_t S = cfg.slots;
    CU(b->lanes.alloc(S * 4));
    // the scratch of the persistent CTAs, not of every slot: a CTA uses it for
    // one block of slots at a time. Each CTA's is one region whose rows hold
    // its BLOCK threads, so a CTA's accesses stay within a few pages (config
    // 4's long searches at half 2048 on B200: 2.08e10 against 2.05e10 keys/s
    // with rows across the whole grid)
    const size_t cta_scratch = (size_t)BLOCK * (2 * (size_t)cfg.max_half + 2) * 4;
    CU(b->scratch.alloc((size_t)b->grid * cta_scratch));
    const std::vector<uint4>& tab = pair_table(cfg.max_half);
    CU(b->table.alloc(tab.size()));
    CU(cudaMemcpy(b->table.p, tab.data(), tab.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    for (uint32_t h = cfg.half; h <= cfg.max_half; h *= 2) {
        std::vector<uint4> pw = pow2_table(base_mult_u64(8ULL * (2ULL * h + 1)), POW2_BITS);
        DevBuf<uint4>& d = b->pow2[h];
        CU(d.alloc(pw.size()));
        CU(cudaMemcpy(d.p, pw.data(), pw.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    }
    b->h_descs.assign(cfg.max_searches, BatchDesc{});
    CU(b->descs.alloc(cfg.max_searches));
    CU(b->pos.alloc(cfg.max_searches));
    CU(b->found.alloc(cfg.max_searches));
    CU(b->mism.alloc(cfg.max_searches));
    CU(b->h_mism.alloc(cfg.max_searches));
    CU(cudaMemset(b->found.p, 0, cfg.max_searches * 4));
    CU(cudaMemset(b->mism.p, 0, cfg.max_searches * 4));
    std::vector<uint4> p8 = pow2_table(base_mult_u64(8), 64);
    CU(b->pow8.alloc(p8.size()));
    CU(cudaMemcpy(b->pow8.p, p8.data(), p8.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    CU(b->blocks.alloc(b->nblocks));
    CU(b->init_list.alloc(b->nblocks));
    CU(b->h_hits.alloc(std::min<uint64_t>(cfg.max_hits, 1u << 16)));
    b->h_blocks.assign(b->nblocks, SlotBlock{NONE, 0});
    for (uint32_t i = 0; i < b->nblocks; i++) b->free_blocks.push_back(b->nblocks - 1 - i);
    for (uint32_t i = 0; i < cfg.max_searches; i++) b->free_sidx.push_back(cfg.max_searches - 1 - i);
    CU(cudaMemcpy(b->descs.p, b->h_descs.data(), cfg.max_searches * sizeof(BatchDesc), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(b->blocks.p, b->h_blocks.data(), b->nblocks * sizeof(SlotBlock), cudaMemcpyHostToDevice));

    for (int fi = 0; fi < FLIGHTS; fi++) {
        Flight& f = b->flights[fi];
        CU(f.counters.alloc(1));
        CU(cudaMemset(f.counters.p, 0, sizeof(Counters)));
        CU(f.surv.alloc(surv_cap));
        CU(f.hits.alloc(cfg.max_hits));
        CU(f.h_counters.alloc(1));
        CU(f.h_descs.alloc(cfg.max_searches));
        CU(f.h_blocks.alloc(b->nblocks));
        CU(f.h_init.alloc(b->nblocks + 1));
        CU(f.h_pos.alloc(cfg.max_searches));
        std::memset(f.h_pos.p, 0, cfg.max_searches * sizeof(SearchPos));
        CU(cudaEventCreate(&f.ev0));
        CU(cudaEventCreate(&f.ev1));
        BatchArgs& a = f.args;
        a.descs = b->descs.p;
        a.blocks = b->blocks.p;
        a.init_list = b->init_list.p;
        a.counters = f.counters.p;
        a.nblocks = b->nblocks;
        a.lanes = b->lanes.p;
        a.scratch = b->scratch.p;
        a.cta_scratch = cta_scratch;
        a.slots = S;
        a.table = b->table.p;
        a.rounds = cfg.rounds;
        a.surv = f.surv.p;
        a.surv_cap = (uint32_t)surv_cap;
        a.hits = f.hits.p;
        a.hit_cap = cfg.max_hits;
        a.pos = b->pos.p;
        a.pow8 = b->pow8.p;
        a.found = b->found.p;
        a.mism = b->mism.p;
        if (cfg.graph != 2) {
            CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_step(b.get(), a, err, errlen);
            cudaError_t ce = rc == OG_OK ? cudaMemcpyAsync(f.h_counters.p, f.counters.p, sizeof(Counters),
                                                           cudaMemcpyDeviceToHost, b->stream)
                                         : cudaSuccess;
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (rc != OG_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            CU(ce);
            CU(e);
            f.graph = g;
            CU(cudaGraphInstantiate(&f.exec, g, 0));
        }
    }
    CU(cudaDeviceSynchronize());
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    b->mem_budget = cfg.memory_budget ? cfg.memory_budget : free_b / 2;
    *out = b.release();
    return OG_OK;
}

int og_batch_admit(og_batch* b, uint64_t search_id, const uint8_t seed[32], const char* filters, uint32_t quota,
                   char* err, size_t errlen) {
    if (!b || !seed || !filters) return fail(err, errlen, OG_E_ARG, "null argument");
    if (b->closed) return fail(err, errlen, OG_E_STATE, "the batch is closed: %s", b->closed_why.c_str());
    if (quota == 0) return fail(err, errlen, OG_E_ARG, "a quota of zero");
    if (b->searches.count(search_id)) return fail(err, errlen, OG_E_STATE, "search %llu is already admitted", (unsigned long long)search_id);
    if (b->free_sidx.empty()) return fail(err, errlen, OG_E_CAPACITY, "%u searches are admitted already", b->cfg.max_searches);
    std::unique_ptr<Search> s(new (std::nothrow) Search());
    if (!s) return fail(err, errlen, OG_E_NOMEM, "host memory");
    s->id = search_id;
    s->quota = quota;
    std::memcpy(s->seed, seed, 32);
    secret_scalar(seed, s->scalar);
    s->start = base_mult(s->scalar);
    // filters: literal prefixes and suffixes
    std::vector<PrefixFilter> fs;
    std::vector<SuffixPattern> sfx;
    std::string why;
    if (!parse_filter_lines(filters, fs, sfx, why)) return fail(err, errlen, OG_E_FILTER, "%s", why.c_str());
    if (fs.empty() && sfx.empty()) return fail(err, errlen, OG_E_FILTER, "no filters");
    if (!fs.empty()) {
        if (!s->fs.build(std::move(fs), 0, why)) return fail(err, errlen, OG_E_FILTER, "%s", why.c_str());
        s->has_prefixes = true;
    }
    if (!sfx.empty()) {
        if (!s->sfx.build(std::move(sfx), 0, why)) return fail(err, errlen, OG_E_FILTER, "%s", why.c_str());
        s->has_suffixes = true;
    }
    const double occupancy = s->fs.occupancy() + s->sfx.occupancy();
    if (occupancy > MAX_OCCUPANCY)
        return fail(err, errlen, OG_E_FILTER, "the filters leave %.1f%% of the index set (at most %.0f%% in a batch)",
                    100 * occupancy, 100 * MAX_OCCUPANCY);
    if (s->has_prefixes)
        for (size_t i = 0; i < s->fs.size(); i++) {
            const PrefixFilter& f = s->fs.filter(i);
            if ((!f.is_pattern() && f.text.size() > FilterSet::DEVICE_SYMBOLS) || f.needs_full_check())
                s->long_filters = true;
        }
    std::vector<uint64_t> keys;
    std::vector<uint32_t> owners, pats;
    if (s->has_prefixes) {
        s->fs.device_tables(s->buckets, keys, owners);
        s->fs.device_patterns(pats);
    }
    if (s->buckets.size() > MAX_BUCKETS) return fail(err, errlen, OG_E_FILTER, "more than %d filter lengths", MAX_BUCKETS);
    std::vector<uint32_t> rows;
    for (size_t j = 0; j < s->sfx.size(); j++) {
        const SuffixPattern& sp = s->sfx.pattern(j);
        std::vector<uint32_t> row(MAX_SUFFIX_SYMBOLS + 1, 0);
        row[0] = (uint32_t)sp.sets.size();
        for (size_t i = 0; i < sp.sets.size(); i++) row[1 + i] = sp.sets[i];
        rows.insert(rows.end(), row.begin(), row.end());
    }
    const size_t words32 = s->fs.words().size() * 2;
    const size_t swords32 = s->sfx.words().size() * 2;
    s->table_bytes = words32 * 4 + keys.size() * 12 + pats.size() * 4 + swords32 * 4 + rows.size() * 4;
    if (b->mem_used + s->table_bytes > b->mem_budget)
        return fail(err, errlen, OG_E_NOMEM, "its tables (%llu bytes) do not fit the remaining budget (%llu of %llu used)",
                    (unsigned long long)s->table_bytes, (unsigned long long)b->mem_used, (unsigned long long)b->mem_budget);
    s->half = choose_half(b, *s);
    s->prob = (double)s->quota / expected_work(*s);
    const auto pw = b->pow2.find(s->half);
    if (pw == b->pow2.end() || !pw->second.p)
        return fail(err, errlen, OG_E_STATE, "no lane-start table for half %u", s->half);
    CU(cudaSetDevice(b->device));
    // the tables come from the batch's pool on the upload stream, so that
    // nothing here waits for a step in flight
    cudaStream_t u = b->ustream;
    if (s->has_prefixes) {
        CU(s->bitmap.alloc(words32, b->pool, u, b->stream));
        CU(s->keys.alloc(keys.size(), b->pool, u, b->stream));
        CU(s->owners.alloc(owners.size(), b->pool, u, b->stream));
        CU(cudaMemcpyAsync(s->bitmap.p, s->fs.words().data(), words32 * 4, cudaMemcpyHostToDevice, u));
        if (!keys.empty()) CU(cudaMemcpyAsync(s->keys.p, keys.data(), keys.size() * 8, cudaMemcpyHostToDevice, u));
        if (!owners.empty()) CU(cudaMemcpyAsync(s->owners.p, owners.data(), owners.size() * 4, cudaMemcpyHostToDevice, u));
        if (!pats.empty()) {
            CU(s->patterns.alloc(pats.size(), b->pool, u, b->stream));
            CU(cudaMemcpyAsync(s->patterns.p, pats.data(), pats.size() * 4, cudaMemcpyHostToDevice, u));
        }
    }
    if (s->has_suffixes) {
        CU(s->sbitmap.alloc(swords32, b->pool, u, b->stream));
        CU(s->suffixes.alloc(rows.size(), b->pool, u, b->stream));
        CU(cudaMemcpyAsync(s->sbitmap.p, s->sfx.words().data(), swords32 * 4, cudaMemcpyHostToDevice, u));
        CU(cudaMemcpyAsync(s->suffixes.p, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, u));
    }
    // wait for the upload stream alone: the copies read pageable host memory,
    // and once they are done any later step may read the tables
    CU(cudaStreamSynchronize(u));
    s->sidx = b->free_sidx.back();
    // its device counters start at zero, after every step launched so far
    CU(cudaMemsetAsync(b->found.p + s->sidx, 0, 4, b->stream));
    CU(cudaMemsetAsync(b->mism.p + s->sidx, 0, 4, b->stream));
    b->free_sidx.pop_back();
    BatchDesc& d = b->h_descs[s->sidx];
    std::memset(&d, 0, sizeof d);
    d.bitmap = s->bitmap.p;
    d.bits = s->fs.bits();
    d.half = s->half;
    d.match = match_tables(s->buckets, s->keys.p, s->owners.p, s->patterns.p,
                           (uint32_t)(pats.size() / FilterSet::PATTERN_ROW));
    d.sbitmap = s->sbitmap.p;
    d.sbits = s->sfx.bits();
    d.prefix_count = s->has_prefixes ? (uint32_t)s->fs.size() : 0;
    d.suffixes = s->suffixes.p;
    d.nsuffix = s->has_suffixes ? (uint32_t)s->sfx.size() : 0;
    // the device may skip a search once it counts its quota, unless some of
    // its hits still need the host's confirmation
    d.quota = s->long_filters ? 0 : quota;
    d.pow2 = pw->second.p;
    d.sx = to_words(s->start.X);
    d.sy = to_words(s->start.Y);
    d.sz = to_words(s->start.Z);
    d.st = to_words(s->start.T);
    if (s->has_suffixes) b->suffix_searches++;
    b->mark(s->sidx);
    s->admit_order = b->admitted++;
    b->mem_used += s->table_bytes;
    b->searches[search_id] = std::move(s);
    b->active_changed = true;
    return OG_OK;
}

size_t og_batch_room(const og_batch* b) { return b ? b->cfg.max_hits : 0; }

int og_batch_step(og_batch* b, og_batch_hit* out, size_t cap, size_t* n, char* err, size_t errlen) {
    if (!b || !n) return fail(err, errlen, OG_E_ARG, "null argument");
    *n = 0;
    b->last_ms = 0;
    b->last_candidates = 0;
    b->last_launches = 0;
    if (b->closed) return fail(err, errlen, OG_E_STATE, "the batch is closed: %s", b->closed_why.c_str());
    CU(cudaSetDevice(b->device));
    while (b->pending() < b->cfg.inflight) {
        bool launched = false;
        const int rc = launch(b, launched, err, errlen);
        if (rc != OG_OK) return close_batch(b, rc, err);
        if (!launched) break;
    }
    if (b->pending() == 0) return OG_OK;
    const int rc = collect(b, out, cap, n, err, errlen);
    if (rc != OG_OK && rc != OG_E_VERIFY && rc != OG_E_CAPACITY) return close_batch(b, rc, err);
    return rc;
}

int og_batch_status(const og_batch* b, uint64_t search_id, og_search_status* st) {
    if (!b || !st) return OG_E_ARG;
    auto it = b->searches.find(search_id);
    if (it == b->searches.end()) return OG_E_STATE;
    const Search& s = *it->second;
    st->windows = s.windows_collected;
    st->candidates = s.windows_collected * (2ULL * s.half + 1);
    st->hits = s.hits.size();
    st->lanes = s.lanes_last;
    st->quota = s.quota;
    st->done = s.done ? 1 : 0;
    st->filters = (uint32_t)(s.fs.size() + s.sfx.size());
    st->table_bytes = s.table_bytes;
    st->status = s.status;
    st->half = s.half;
    return OG_OK;
}

int og_batch_results(const og_batch* b, uint64_t search_id, og_batch_hit* out, size_t cap, size_t* n) {
    if (!b || !n) return OG_E_ARG;
    *n = 0;
    auto it = b->searches.find(search_id);
    if (it == b->searches.end()) return OG_E_STATE;
    const Search& s = *it->second;
    if (cap < s.hits.size()) return OG_E_CAPACITY;
    for (size_t i = 0; i < s.hits.size(); i++) out[i] = s.hits[i];
    *n = s.hits.size();
    return OG_OK;
}

int og_batch_retire(og_batch* b, uint64_t search_id) {
    if (!b) return OG_E_ARG;
    auto it = b->searches.find(search_id);
    if (it == b->searches.end()) return OG_E_STATE;
    Search& s = *it->second;
    cudaSetDevice(b->device);
    release_blocks(b, s);
    b->free_sidx.push_back(s.sidx);
    b->mem_used -= s.table_bytes;
    if (s.has_suffixes) b->suffix_searches--;
    if (!s.done) b->active_changed = true;
    // its tables go back to the pool after the steps already launched
    b->searches.erase(it);
    return OG_OK;
}

void og_batch_counts(const og_batch* b, size_t* admitted, size_t* running) {
    size_t a = 0, r = 0;
    if (b)
        for (const auto& kv : b->searches) {
            a++;
            if (!kv.second->done) r++;
        }
    if (admitted) *admitted = a;
    if (running) *running = r;
}

float og_batch_last_step_ms(const og_batch* b) { return b ? b->last_ms : 0.f; }
uint64_t og_batch_last_step_candidates(const og_batch* b) { return b ? b->last_candidates : 0; }
uint32_t og_batch_last_step_launches(const og_batch* b) { return b ? b->last_launches : 0; }

void og_batch_memory(const og_batch* b, uint64_t* used, uint64_t* budget) {
    if (used) *used = b ? b->mem_used : 0;
    if (budget) *budget = b ? b->mem_budget : 0;
}

void og_batch_shape(const og_batch* b, og_batch_config* cfg) {
    if (b && cfg) *cfg = b->cfg;
}

int og_batch_tune(int ordinal, uint32_t searches, float max_step_ms, og_batch_config* out, double* keys_per_s,
                  char* err, size_t errlen) {
    if (!out) return fail(err, errlen, OG_E_ARG, "null argument");
    if (searches == 0) searches = 64;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(err, errlen, OG_E_NODEVICE, "no CUDA device is available");
    if (ordinal < 0 || ordinal >= count) return fail(err, errlen, OG_E_ARG, "device %d of %d", ordinal, count);
    CU(cudaSetDevice(ordinal));
    int per_sm = 0, sms = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_search_kernel, BLOCK, STAGED_BYTES));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ordinal));
    const uint32_t fit = (uint32_t)std::max(1, per_sm);
    // a mix that never finishes: each search one ten-symbol prefix (50 bits)
    std::vector<std::string> prefixes(searches);
    for (uint32_t j = 0; j < searches; j++) {
        std::string p;
        uint32_t v = j * 2654435761u + 12345u;
        for (int k = 0; k < 10; k++) {
            p.push_back(BASE32_ALPHABET[v & 31]);
            v = v * 1103515245u + 12345u;
        }
        prefixes[j] = p;
    }
    og_batch_config best{};
    double best_rate = -1;
    int last = OG_E_DEVICE;
    for (uint32_t half : {128u, 256u, 512u}) {
        for (uint32_t grid : {fit, std::max(1u, fit / 2)}) {
            for (uint32_t waves : {1u, 2u, 3u}) {
                og_batch_config c{};
                c.half = half;
                c.grid = grid;
                c.slots = waves * grid * (uint32_t)sms * BLOCK;
                c.rounds = 1;
                c.max_searches = searches;
                c.graph = 1;
                og_batch* b = nullptr;
                last = og_batch_new(ordinal, &c, &b, err, errlen);
                if (last != OG_OK) continue;
                for (uint32_t j = 0; j < searches && last == OG_OK; j++) {
                    uint8_t seed[32] = {0};
                    const uint32_t id = 0x7f000000u + j;
                    std::memcpy(seed, &id, 4);
                    last = og_batch_admit(b, j, seed, prefixes[j].c_str(), 1, err, errlen);
                }
                double ms = 0, cand = 0;
                for (int step = 0; step < 6 && last == OG_OK; step++) {
                    size_t n = 0;
                    last = og_batch_step(b, nullptr, 0, &n, err, errlen);
                    if (step >= 2) {
                        ms += og_batch_last_step_ms(b);
                        cand += (double)og_batch_last_step_candidates(b);
                    }
                }
                og_batch_free(b);
                if (last != OG_OK || ms <= 0) continue;
                const double rate = cand / (ms * 1e-3);
                if ((max_step_ms <= 0 || ms / 4 <= max_step_ms) && rate > best_rate) {
                    best_rate = rate;
                    best = og_batch_config{};
                    best.half = half;
                    best.slots = c.slots;
                    best.rounds = 1;
                    best.grid = grid;
                }
            }
        }
    }
    if (best_rate < 0) return fail(err, errlen, last, "no batch shape ran within %.1f ms a step", max_step_ms);
    Shape s;
    s.first = best.half;
    s.second = best.slots;
    s.block = best.grid;
    s.rounds = best.rounds;
    s.rate = best_rate;
    s.at = unix_now();
    tuning_put(batch_key(ordinal), s);
    *out = best;
    if (keys_per_s) *keys_per_s = best_rate;
    return OG_OK;
}

int og_batch_plant_mismatch(og_batch* b, uint64_t search_id) {
    if (!b) return OG_E_ARG;
    if (!b->searches.count(search_id)) return OG_E_STATE;
    b->planted.insert(search_id);
    return OG_OK;
}

void og_batch_free(og_batch* b) { delete b; }

}  // extern "C"
