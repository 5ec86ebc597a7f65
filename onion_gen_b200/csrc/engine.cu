// og_engine: the single-search device engine behind the C ABI.
//
// Mirrors cuda::Engine (src/gpu/cuda.rs:103-365) and the shape logic of
// gpu::Engine (src/gpu/mod.rs:292-477): host precompute once, lane state
// resident in HBM, one persistent kernel launch per advance, a copy of only
// the survivors that were written, and an overflow that is an error rather
// than a truncation. Two advances can be in flight, each with its own record
// buffers, so that one advance's survivors cross back and are checked while
// the next one runs. The device match (og_engine_match_on_device, and the
// filter engine of og_engine_new_filters) adds one kernel per advance.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/onion_gen_b200.h"
#include "host/common.h"
#include "host/filters.h"
#include "host/tuning.h"
#include "kernels.cuh"

#ifndef OG_LB_THREADS
#define OG_LB_THREADS 128
#endif

using namespace og;

namespace og {

// Affine x, y of many points with one inversion (Montgomery).
static void batch_affine(const std::vector<Pt>& pts, std::vector<F51>& xs, std::vector<F51>& ys) {
    const size_t n = pts.size();
    std::vector<F51> prefix(n);
    F51 run = f_one();
    for (size_t i = 0; i < n; i++) {
        prefix[i] = run;
        run = f_mul(run, pts[i].Z);
    }
    F51 inv = f_inv(run);
    xs.resize(n);
    ys.resize(n);
    for (size_t i = n; i-- > 0;) {
        const F51 zi = f_mul(inv, prefix[i]);
        inv = f_mul(inv, pts[i].Z);
        xs[i] = f_mul(pts[i].X, zi);
        ys[i] = f_mul(pts[i].Y, zi);
    }
}

// The table Q_m = 8m G, m = 1..half, affine (x, y, xy), in the device
// layout; the same for every search, so built once per half.
const std::vector<uint4>& pair_table(uint32_t half) {
    static std::mutex mu;
    static std::map<uint32_t, std::unique_ptr<std::vector<uint4>>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(half);
    if (it != cache.end()) return *it->second;
    std::vector<Pt> pts(half);
    const Pt eight = base_mult_u64(8);
    Pt p = eight;
    for (uint32_t m = 0; m < half; m++) {
        pts[m] = p;
        p = pt_add(p, eight);
    }
    std::vector<F51> xs, ys;
    batch_affine(pts, xs, ys);
    auto v = std::make_unique<std::vector<uint4>>((size_t)half * 6);
    for (uint32_t m = 0; m < half; m++) {
        uint4* d = v->data() + (size_t)m * 6;
        put_fe(d + 0, 1, xs[m]);
        put_fe(d + 2, 1, ys[m]);
        put_fe(d + 4, 1, f_mul(xs[m], ys[m]));
    }
    auto& ref = *v;
    cache[half] = std::move(v);
    return ref;
}

// 2^k * stride for k < nbits in cached form (y+x, y-x, 2dxy), device layout.
std::vector<uint4> pow2_table(const Pt& stride, uint32_t nbits) {
    std::vector<uint4> out((size_t)std::max<uint32_t>(nbits, 1) * 6);
    Pt p = stride;
    for (uint32_t k = 0; k < nbits; k++) {
        const Niels c = pt_niels(p);
        uint4* d = out.data() + (size_t)k * 6;
        put_fe(d + 0, 1, c.ypx);
        put_fe(d + 2, 1, c.ymx);
        put_fe(d + 4, 1, c.xy2d);
        p = pt_dbl(p);
    }
    return out;
}

uint32_t bits_for(uint64_t v) {
    uint32_t b = 0;
    while (b < 64 && (v >> b) != 0) b++;
    return b;
}

static_assert(FilterSet::PATTERN_ROW == PATTERN_WORDS, "pattern rows: host and device layouts agree");

MatchTables match_tables(const std::vector<FilterSet::DeviceBucket>& buckets, const uint64_t* keys,
                         const uint32_t* owners, const uint32_t* patterns, uint32_t npatterns) {
    MatchTables t{};
    t.keys = keys;
    t.owners = owners;
    t.patterns = patterns;
    t.npatterns = npatterns;
    t.nbuckets = (uint32_t)std::min<size_t>(buckets.size(), MAX_MATCH_BUCKETS);
    for (uint32_t i = 0; i < t.nbuckets; i++) {
        t.bucket_bits[i] = buckets[i].bits;
        t.bucket_off[i] = buckets[i].offset;
        t.bucket_len[i] = buckets[i].count;
    }
    return t;
}

// FNV-1a over the words of a bitmap: identifies the bitmap an engine was
// built with, so that a filter set handed in later can be checked against it.
uint64_t words_hash(const uint64_t* w, size_t n) {
    uint64_t h = 0xcbf29ce484222325ULL;
    for (size_t i = 0; i < n; i++) {
        uint64_t v = w[i];
        for (int k = 0; k < 8; k++) {
            h ^= v & 0xff;
            h *= 0x100000001b3ULL;
            v >>= 8;
        }
    }
    return h;
}

}  // namespace og

struct og_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    og_engine_config cfg{};
    uint32_t slots = 0;
    uint32_t bits = 0;
    uint32_t grid = 0;  // persistent CTAs of the paired kernel
    size_t cap = 0;
    uint64_t launches = 0;
    float last_ms = 0;
    bool overflowed = false;
    DevBuf<uint4> lanes, scratch, table, pow2;
    DevBuf<uint32_t> bitmap;
    // Two advances can be in flight (og_engine_launch / og_engine_collect):
    // each has its own record buffers and counters, so the host can read one
    // advance's results while the next one runs; the lanes and the scratch
    // are shared, the launches being ordered on one stream.
    struct Flight {
        DevBuf<uint32_t> counts;  // survivors, matches, mismatched suffix keys
        DevBuf<HitRec> hits;
        DevBuf<MatchRec> matches;
        HostBuf<uint32_t> h_counts;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
        uint64_t launch = 0;
        bool match = false;
    } fl[2];
    uint32_t head = 0, inflight = 0;
    cudaStream_t cstream = nullptr;  // record copies, beside the next advance's kernels
    HostBuf<HitRec> h_recs;  // pinned: survivors, or (as MatchRec, the same size) matches
    static constexpr int COPY_CHUNKS = 16;
    cudaEvent_t chunk_ev[COPY_CHUNKS] = {};  // a chunk of the records has reached h_recs
    PairedArgs pa{};
    ChainArgs ca{};
    uint64_t bitmap_hash = 0;  // of the bitmap the engine was created with
    DevBuf<uint32_t> sbitmap;  // suffix bitmap (og_engine_new_filters)
    uint32_t sbits = 0;
    Pt start{};
    // device exact match (og_engine_match_on_device)
    bool matching = false;
    bool long_filters = false;  // some filter is longer than the device tables reach
    uint32_t prefix_count = 0;
    og::FilterSet fs;
    DevBuf<uint64_t> mkeys;
    DevBuf<uint32_t> mowners, mpatterns;
    DevBuf<uint32_t> suffixes;
    DevBuf<uint4> pow8;
    MatchArgs ma{};

    ~og_engine() {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        if (cstream) {
            cudaStreamSynchronize(cstream);
            cudaStreamDestroy(cstream);
        }
        for (Flight& f : fl) {
            if (f.ev0) cudaEventDestroy(f.ev0);
            if (f.ev1) cudaEventDestroy(f.ev1);
            if (f.done) cudaEventDestroy(f.done);
        }
        for (cudaEvent_t ev : chunk_ev)
            if (ev) cudaEventDestroy(ev);
    }
};

namespace {

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            return fail(err, errlen, _e == cudaErrorMemoryAllocation ? OG_E_NOMEM : OG_E_DEVICE, \
                        "%s: %s", #call, cuda_text(_e).c_str());                              \
    } while (0)

// Lanes one wave of the search kernel holds: resident CTAs x block x lanes
// per thread.
int resident_lanes(int device, uint32_t scheme, uint32_t half, uint32_t block, uint32_t* out, char* err,
                   size_t errlen, uint32_t lanes_per_thread = 1) {
    KernelInfo info{};
    cudaError_t e = scheme == OG_SCHEME_CHAIN ? chain_info((int)block, &info)
                                              : paired_info((int)block, half, lanes_per_thread, &info);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "kernel attributes: %s", cuda_text(e).c_str());
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "device attributes: %s", cuda_text(e).c_str());
    *out = (uint32_t)std::max(1, info.blocks_per_sm) * (uint32_t)sms * block * lanes_per_thread;
    return OG_OK;
}

// Records one advance may produce: every candidate in dump mode; else what
// the bitmaps' measured occupancy lets through, plus eight standard
// deviations of its binomial spread, plus a floor. For uniform keys each
// candidate survives with exactly that probability, so the margin is not
// crossed in practice, and an overflow is still an error, never a
// truncation. (src/gpu/mod.rs:298-312 sizes the room from one slot per
// prefix, which short prefixes overflow; this takes the real occupancy.)
size_t room_for(uint64_t batch, bool dump, double occupancy) {
    if (dump) return (size_t)batch;
    const double expected = (double)batch * occupancy;
    const double want = expected + 8.0 * std::sqrt(expected) + 1024.0;
    return (size_t)std::min<double>((double)batch, std::max(4096.0, want));
}

// Bitmaps that let more than this share of candidates through get the
// paired kernel that stages survivor records per warp (one atomic per 32
// records): on B200 the direct append ran 21.0 G keys/s at 1.5e-5 and 19.2
// at 5.2e-2 of candidates surviving, the staged one a flat 20.4, and they
// cross near 6e-3.
constexpr double STAGE_OCCUPANCY = 6e-3;

// Expected survivors of one advance that the default shape allows: 2^26
// records, 3.2 GB of records per advance in flight.
constexpr double SURVIVOR_BUDGET = (double)(1u << 26);

// `f` (may be null) supplies both bitmaps instead of `bitmap`: its prefix
// index (if it has prefixes) and its suffix index (if it has suffixes).
int build_engine(int ordinal, const uint8_t start[128], og_engine_config cfg, const uint64_t* bitmap, size_t words,
                 uint32_t bits, og_engine** out, char* err, size_t errlen, const og_filters* f = nullptr) {
    if (!out || !start) return fail(err, errlen, OG_E_ARG, "null argument");
    *out = nullptr;
    const bool suffixed = f && f->has_suffixes;
    if (f) {
        if (cfg.dump) return fail(err, errlen, OG_E_ARG, "a filter engine cannot keep every candidate (dump)");
        bitmap = f->has_prefixes ? f->set.words().data() : nullptr;
        words = f->has_prefixes ? f->set.words().size() : 0;
        bits = f->has_prefixes ? f->set.bits() : 0;
    }
    if (cfg.scheme > OG_SCHEME_CHAIN) return fail(err, errlen, OG_E_ARG, "unknown scheme %u", cfg.scheme);
    if (cfg.lanes_per_thread > 2 || (cfg.scheme == OG_SCHEME_CHAIN && cfg.lanes_per_thread > 1))
        return fail(err, errlen, OG_E_ARG, "%u lanes per thread (the paired scheme takes 1 or 2, the chain 1)",
                    cfg.lanes_per_thread);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(err, errlen, OG_E_NODEVICE, "no CUDA device is available");
    if (ordinal < 0 || ordinal >= count) return fail(err, errlen, OG_E_ARG, "device %d of %d", ordinal, count);
    if (!cfg.dump && (bitmap || !suffixed)) {
        if (!bitmap) return fail(err, errlen, OG_E_ARG, "no bitmap: without one every candidate would cross back");
        if (bits < 8 || bits > 32) return fail(err, errlen, OG_E_ARG, "bitmap width %u outside 8..32", bits);
        const size_t need = (size_t)(((1ULL << bits) + 63) / 64);
        if (words < need) return fail(err, errlen, OG_E_ARG, "%zu words for a %u-bit index (%zu needed)", words, bits, need);
    }
    CU(cudaSetDevice(ordinal));
    if (cfg.block == 0) cfg.block = 128;
    if (cfg.block % 32 || cfg.block > OG_LB_THREADS)
        return fail(err, errlen, OG_E_ARG, "block %u (a multiple of 32, at most %d)", cfg.block, OG_LB_THREADS);
    if (cfg.lanes_per_thread == 0) cfg.lanes_per_thread = 1;
    const uint32_t lpt = cfg.lanes_per_thread;
    const bool auto_half = cfg.half == 0;
    if (cfg.half == 0) cfg.half = cfg.scheme == OG_SCHEME_CHAIN ? 1024 : 2048;
    if (cfg.scheme == OG_SCHEME_PAIRED && cfg.half > 2048) return fail(err, errlen, OG_E_ARG, "half %u > 2048", cfg.half);
    if (cfg.scheme == OG_SCHEME_CHAIN && cfg.half > 65536) return fail(err, errlen, OG_E_ARG, "n %u > 65536", cfg.half);
    double occ = 1.0;  // the share of candidates the bitmaps let through
    if (!cfg.dump) {
        occ = 0.0;
        if (bitmap) {
            std::vector<uint64_t> w(bitmap, bitmap + (size_t)(((1ULL << bits) + 63) / 64));
            occ = bitmap_occupancy(w, bits);
        }
        if (suffixed) occ += f->suffixes.occupancy();
    }
    if (cfg.lanes == 0) {
        uint32_t resident = 0;
        int rc = resident_lanes(ordinal, cfg.scheme, cfg.half, cfg.block, &resident, err, errlen, lpt);
        if (rc) return rc;
        if (cfg.scheme == OG_SCHEME_PAIRED) {
            // the persistent kernel takes lanes a block at a time: eight
            // blocks per resident CTA leave the last ones little tail
            // (measured +3.5% over two), while the scratch stays that of the
            // resident CTAs. When one advance would return more than the
            // survivor budget, a shorter inversion batch comes first (config
            // 3's 5 % survivors on B200: half 512 at eight waves 19.2 G keys/s,
            // half 2048 at one wave 16.6), then fewer waves.
            uint32_t waves = 8;
            const auto expected = [&] { return (double)resident * waves * (2.0 * cfg.half + 1) * occ; };
            while (auto_half && cfg.half > 256 && expected() > SURVIVOR_BUDGET) cfg.half /= 2;
            while (waves > 1 && expected() > SURVIVOR_BUDGET) waves /= 2;
            cfg.lanes = resident * waves;
        } else {
            // persistent too: four waves of resident blocks (on B200 at
            // n = 1024: 9.05 G keys/s for the earlier one-lane-per-thread
            // kernel at two waves; persistent, over two runs, 9.19-9.25 /
            // 9.31-9.37 / 9.20-9.54 at 2 / 4 / 8 waves, all on the scratch
            // of one wave)
            cfg.lanes = resident * 4;
        }
    }
    const uint32_t slots = cfg.scheme == OG_SCHEME_CHAIN ? cfg.half : 2 * cfg.half + 1;
    cfg.lanes = (cfg.lanes + cfg.block * lpt - 1) / (cfg.block * lpt) * (cfg.block * lpt);
    if (cfg.lanes > (1u << 24)) return fail(err, errlen, OG_E_ARG, "%u lanes (at most 2^24)", cfg.lanes);
    if (cfg.rounds == 0) {
        const uint64_t per_round = (uint64_t)cfg.lanes * slots;
        cfg.rounds = (uint32_t)std::max<uint64_t>(1, (1ULL << 27) / per_round);
    }
    const double occupancy = occ;
    // keep the expected survivors of one advance within the budget
    while (!cfg.dump && cfg.rounds > 1 && (double)cfg.lanes * slots * cfg.rounds * occupancy > SURVIVOR_BUDGET)
        cfg.rounds /= 2;
    if ((uint64_t)cfg.rounds * slots > 0xffffffffULL) return fail(err, errlen, OG_E_ARG, "too many rounds per advance");

    Pt start_pt = point_from_bytes(start);
    if (!point_valid(start_pt)) return fail(err, errlen, OG_E_ARG, "the start point is not on the curve");

    std::unique_ptr<og_engine> e(new (std::nothrow) og_engine());
    if (!e) return fail(err, errlen, OG_E_NOMEM, "host memory");
    e->device = ordinal;
    e->cfg = cfg;
    e->slots = slots;
    e->bits = bits;
    CU(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&e->cstream, cudaStreamNonBlocking));
    for (og_engine::Flight& f : e->fl) {
        CU(cudaEventCreate(&f.ev0));
        CU(cudaEventCreate(&f.ev1));
        CU(cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming));
    }
    for (cudaEvent_t& ev : e->chunk_ev) CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));

    const size_t L = cfg.lanes;
    const uint64_t batch = (uint64_t)L * slots * cfg.rounds;
    e->cap = cfg.room ? cfg.room : room_for(batch, cfg.dump != 0, occupancy);
    e->cfg.room = (uint32_t)std::min<size_t>(e->cap, 0xffffffffu);
    const uint32_t coords = cfg.scheme == OG_SCHEME_CHAIN ? 4 : 2;
    CU(e->lanes.alloc(L * coords * 2));
    const size_t elems = cfg.scheme == OG_SCHEME_CHAIN ? cfg.half : 2 * (size_t)cfg.half + 2;
    {
        // both kernels are persistent: scratch for the resident CTAs only
        // (the chain kernel's no more CTAs than blocks of lanes)
        uint32_t resident = 0;
        int rc = resident_lanes(ordinal, cfg.scheme, cfg.half, cfg.block, &resident, err, errlen, lpt);
        if (rc) return rc;
        e->grid = std::max<uint32_t>(1, resident / (cfg.block * lpt));
        if (cfg.scheme == OG_SCHEME_CHAIN) e->grid = std::min<uint32_t>(e->grid, (uint32_t)(L / cfg.block));
        // one scratch column per lane a thread holds; a chain CTA's rows hold
        // CHAIN_ROW threads whatever its block
        const size_t row = cfg.scheme == OG_SCHEME_CHAIN ? CHAIN_ROW : (size_t)cfg.block * lpt;
        CU(e->scratch.alloc((size_t)e->grid * row * elems * 4));
    }
    for (og_engine::Flight& f : e->fl) {
        CU(f.counts.alloc(4));
        CU(f.hits.alloc(e->cap));
        CU(f.h_counts.alloc(4));
    }
    CU(e->h_recs.alloc(e->cap));
    if (!cfg.dump && bitmap) {
        const size_t w32 = (size_t)(((1ULL << bits) + 31) / 32);
        CU(e->bitmap.alloc(std::max<size_t>(w32, 2)));
        CU(cudaMemcpyAsync(e->bitmap.p, bitmap, w32 * 4, cudaMemcpyHostToDevice, e->stream));
        e->bitmap_hash = words_hash(bitmap, (size_t)(((1ULL << bits) + 63) / 64));
    }
    if (suffixed) {
        const uint32_t sb = f->suffixes.bits();
        const size_t w32 = (size_t)(((1ULL << sb) + 31) / 32);
        CU(e->sbitmap.alloc(std::max<size_t>(w32, 2)));
        CU(cudaMemcpyAsync(e->sbitmap.p, f->suffixes.words().data(), w32 * 4, cudaMemcpyHostToDevice, e->stream));
        e->sbits = sb;
    }
    e->start = start_pt;

    // lane start points
    InitArgs ia{};
    Pt base, stride;
    if (cfg.scheme == OG_SCHEME_PAIRED) {
        base = pt_add(start_pt, base_mult_u64(8ULL * (cfg.half + 1)));  // first centre
        stride = base_mult_u64(8ULL * slots);
        ia.affine_out = 1;
    } else {
        base = start_pt;
        stride = base_mult_u64(8ULL * slots);
        ia.affine_out = 0;
    }
    const uint32_t nbits = bits_for(L - 1);
    std::vector<uint4> pw = pow2_table(stride, nbits);
    CU(e->pow2.alloc(pw.size()));
    CU(cudaMemcpyAsync(e->pow2.p, pw.data(), pw.size() * sizeof(uint4), cudaMemcpyHostToDevice, e->stream));
    ia.lanes = e->lanes.p;
    ia.bx = to_words(base.X);
    ia.by = to_words(base.Y);
    ia.bz = to_words(base.Z);
    ia.bt = to_words(base.T);
    ia.pow2 = e->pow2.p;
    ia.nbits = nbits;
    ia.lanes_n = cfg.lanes;
    CU(launch_init(ia, 128, e->stream));

    if (cfg.scheme == OG_SCHEME_PAIRED) {
        const std::vector<uint4>& tab = pair_table(cfg.half);
        CU(e->table.alloc(tab.size()));
        CU(cudaMemcpyAsync(e->table.p, tab.data(), tab.size() * sizeof(uint4), cudaMemcpyHostToDevice, e->stream));
        F51 wx, wy;
        pt_affine(base_mult_u64(8ULL * slots * L), wx, wy);
        PairedArgs& a = e->pa;
        a.table = e->table.p;
        a.lanes = e->lanes.p;
        a.scratch = e->scratch.p;
        a.work = nullptr;  // the flight's counter, set per launch
        a.slots_n = e->grid * cfg.block * lpt;
        a.lanes_per_thread = lpt;
        a.stage_records = (!cfg.dump && lpt == 1 && occupancy > STAGE_OCCUPANCY) ? 1u : 0u;
        a.bitmap = cfg.dump ? nullptr : e->bitmap.p;
        a.bits = bits;
        a.sbitmap = e->sbitmap.p;
        a.sbits = e->sbits;
        a.hits = nullptr;     // set per launch to the flight's buffers
        a.counter = nullptr;
        a.cap = (uint32_t)std::min<size_t>(e->cap, 0xffffffffu);
        a.search = 0;
        a.wx = to_words(wx);
        a.wy = to_words(wy);
        a.wt = to_words(f_mul(wx, wy));
        a.lanes_n = cfg.lanes;
        a.half = cfg.half;
        a.rounds = cfg.rounds;
    } else {
        const Niels step = pt_niels(base_mult_u64(8));
        ChainArgs& a = e->ca;
        a.lanes = e->lanes.p;
        a.scratch = e->scratch.p;
        a.work = nullptr;  // the flight's counter, set per launch
        a.slots_n = e->grid * cfg.block;
        a.bitmap = cfg.dump ? nullptr : e->bitmap.p;
        a.bits = bits;
        a.sbitmap = e->sbitmap.p;
        a.sbits = e->sbits;
        a.hits = nullptr;     // set per launch to the flight's buffers
        a.counter = nullptr;
        a.cap = (uint32_t)std::min<size_t>(e->cap, 0xffffffffu);
        a.search = 0;
        a.step_ypx = to_words(step.ypx);
        a.step_ymx = to_words(step.ymx);
        a.step_t2d = to_words(step.xy2d);
        if (L > 1) {
            const Niels jump = pt_niels(base_mult_u64(8ULL * (L - 1) * slots));
            a.jump_ypx = to_words(jump.ypx);
            a.jump_ymx = to_words(jump.ymx);
            a.jump_t2d = to_words(jump.xy2d);
        }
        a.lanes_n = cfg.lanes;
        a.n = cfg.half;
        a.rounds = cfg.rounds;
    }
    CU(cudaStreamSynchronize(e->stream));
    *out = e.release();
    return OG_OK;
}

// One advance timed on the device, candidates per second (the method of
// gpu::Engine::time_one_launch, src/gpu/mod.rs:420-428, on CUDA events).
double time_advance(og_engine* e, std::vector<og_survivor>& buf) {
    size_t n = 0;
    if (og_engine_advance(e, buf.data(), buf.size(), &n, nullptr, 0) != OG_OK) return -1;
    if (og_engine_advance(e, buf.data(), buf.size(), &n, nullptr, 0) != OG_OK) return -1;
    const double ms = e->last_ms;
    return ms > 0 ? (double)og_engine_batch(e) / (ms * 1e-3) : -1;
}


// Device exact match for `f`: prefix tables, suffix patterns, the table of
// 2^j 8G the suffix confirmation walks, and the match buffers.
int enable_matching(og_engine* e, const og_filters* f, char* err, size_t errlen) {
    std::vector<FilterSet::DeviceBucket> buckets;
    std::vector<uint64_t> keys;
    std::vector<uint32_t> owners, pats;
    if (f->has_prefixes) {
        f->set.device_tables(buckets, keys, owners);
        f->set.device_patterns(pats);
    }
    if (buckets.size() > (size_t)MAX_MATCH_BUCKETS)
        return fail(err, errlen, OG_E_FILTER, "more than %d filter lengths", MAX_MATCH_BUCKETS);
    std::vector<uint32_t> sfx;
    if (f->has_suffixes) {
        for (size_t j = 0; j < f->suffixes.size(); j++) {
            const SuffixPattern& p = f->suffixes.pattern(j);
            std::vector<uint32_t> row(MAX_SUFFIX_SYMBOLS + 1, 0);
            row[0] = (uint32_t)p.sets.size();
            for (size_t i = 0; i < p.sets.size(); i++) row[1 + i] = p.sets[i];
            sfx.insert(sfx.end(), row.begin(), row.end());
        }
    }
    e->matching = false;
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->stream));
    CU(e->mkeys.alloc(std::max<size_t>(keys.size(), 1)));
    CU(e->mowners.alloc(std::max<size_t>(owners.size(), 1)));
    if (!keys.empty()) {
        CU(cudaMemcpyAsync(e->mkeys.p, keys.data(), keys.size() * 8, cudaMemcpyHostToDevice, e->stream));
        CU(cudaMemcpyAsync(e->mowners.p, owners.data(), owners.size() * 4, cudaMemcpyHostToDevice, e->stream));
    }
    if (!pats.empty()) {
        CU(e->mpatterns.alloc(pats.size()));
        CU(cudaMemcpyAsync(e->mpatterns.p, pats.data(), pats.size() * 4, cudaMemcpyHostToDevice, e->stream));
    }
    std::vector<uint4> pw;
    if (!sfx.empty()) {
        CU(e->suffixes.alloc(sfx.size()));
        CU(cudaMemcpyAsync(e->suffixes.p, sfx.data(), sfx.size() * 4, cudaMemcpyHostToDevice, e->stream));
        pw = pow2_table(base_mult_u64(8), 64);
        CU(e->pow8.alloc(pw.size()));
        CU(cudaMemcpyAsync(e->pow8.p, pw.data(), pw.size() * sizeof(uint4), cudaMemcpyHostToDevice, e->stream));
    }
    for (og_engine::Flight& fl : e->fl) CU(fl.matches.alloc(e->cap));
    CU(cudaStreamSynchronize(e->stream));
    e->fs = f->set;
    e->long_filters = false;
    if (f->has_prefixes)
        for (size_t i = 0; i < e->fs.size(); i++)
            if (!e->fs.filter(i).is_pattern() && e->fs.filter(i).text.size() > FilterSet::DEVICE_SYMBOLS)
                e->long_filters = true;
    e->prefix_count = f->has_prefixes ? (uint32_t)f->set.size() : 0;
    MatchArgs& m = e->ma;
    m = MatchArgs{};
    m.surv = nullptr;  // the flight's buffers, set per launch
    m.surv_count = nullptr;
    m.surv_cap = (uint32_t)std::min<size_t>(e->cap, 0xffffffffu);
    m.t = match_tables(buckets, e->mkeys.p, e->mowners.p, e->mpatterns.p,
                       (uint32_t)(pats.size() / FilterSet::PATTERN_ROW));
    m.sbitmap = sfx.empty() ? nullptr : e->sbitmap.p;
    m.sbits = e->sbits;
    m.suffixes = e->suffixes.p;
    m.nsuffix = f->has_suffixes ? (uint32_t)f->suffixes.size() : 0;
    m.prefix_count = e->prefix_count;
    m.sx = to_words(e->start.X);
    m.sy = to_words(e->start.Y);
    m.sz = to_words(e->start.Z);
    m.st = to_words(e->start.T);
    m.pow8 = e->pow8.p;
    m.lanes = e->cfg.lanes;
    m.slots = e->slots;
    m.paired = e->cfg.scheme == OG_SCHEME_PAIRED ? 1u : 0u;
    m.out = nullptr;
    m.out_count = nullptr;
    m.out_cap = m.surv_cap;
    m.mismatch = nullptr;
    e->matching = true;
    return OG_OK;
}


// One advance onto the engine's stream, into the next free flight: the
// search kernel, optionally the device match, and the copy of the counters.
int enqueue_advance(og_engine* e, bool match, char* err, size_t errlen) {
    if (!e) return fail(err, errlen, OG_E_ARG, "null argument");
    if (e->overflowed) return fail(err, errlen, OG_E_STATE, "an earlier advance overflowed; the engine is closed");
    if (e->inflight == 2) return fail(err, errlen, OG_E_STATE, "two advances are in flight: collect one first");
    og_engine::Flight& f = e->fl[(e->head + e->inflight) & 1];
    CU(cudaSetDevice(e->device));
    CU(cudaMemsetAsync(f.counts.p, 0, 4 * sizeof(uint32_t), e->stream));
    CU(cudaEventRecord(f.ev0, e->stream));
    if (e->cfg.scheme == OG_SCHEME_PAIRED) {
        e->pa.hits = f.hits.p;
        e->pa.counter = f.counts.p;
        e->pa.work = f.counts.p + 3;
        CU(launch_paired(e->pa, (int)e->cfg.block, (int)e->grid, e->stream));
    } else {
        e->ca.hits = f.hits.p;
        e->ca.counter = f.counts.p;
        e->ca.work = f.counts.p + 3;
        CU(launch_chain(e->ca, (int)e->cfg.block, (int)e->grid, e->stream));
    }
    CU(cudaEventRecord(f.ev1, e->stream));
    if (match) {
        MatchArgs& m = e->ma;
        m.surv = f.hits.p;
        m.surv_count = f.counts.p;
        m.out = f.matches.p;
        m.out_count = f.counts.p + 1;
        m.mismatch = f.counts.p + 2;
        m.window0 = e->launches * (uint64_t)e->cfg.rounds * e->cfg.lanes;
        int sms = 0;
        CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
        CU(launch_match(m, std::max(sms, 1) * 4, e->stream));
    }
    CU(cudaMemcpyAsync(f.h_counts.p, f.counts.p, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream));
    CU(cudaEventRecord(f.done, e->stream));
    f.launch = e->launches++;
    f.match = match;
    e->inflight++;
    return OG_OK;
}

// Host threads that convert n records: up to 16 when n is large enough
// (2^20 records) for the threads to pay.
size_t host_workers(size_t n) {
    return n >= (1u << 20) ? std::min<size_t>(16, std::max(1u, std::thread::hardware_concurrency())) : 1;
}

// Waits for the oldest flight and checks its counts. The flight is released
// whatever happens; its records (HitRec survivors, or MatchRec matches for a
// matching flight) are left on the device for copy_records, at *src.
int collect_flight(og_engine* e, bool match, uint32_t* count, uint64_t* launch, const void** src, char* err,
                   size_t errlen) {
    if (e->inflight == 0) return fail(err, errlen, OG_E_STATE, "no advance in flight");
    og_engine::Flight& f = e->fl[e->head];
    if (f.match != match)
        return fail(err, errlen, OG_E_STATE, "the oldest advance in flight was launched %s the device match",
                    f.match ? "with" : "without");
    e->head ^= 1;
    e->inflight--;
    CU(cudaSetDevice(e->device));
    CU(cudaEventSynchronize(f.done));
    cudaEventElapsedTime(&e->last_ms, f.ev0, f.ev1);
    *launch = f.launch;
    const uint32_t found = f.h_counts.p[0];
    if (found > e->cap) {
        e->overflowed = true;
        return fail(err, errlen, OG_E_OVERFLOW,
                    "one advance produced %u survivors and only %zu fit; the index is too narrow for what it "
                    "is filtering: a wider index is the answer",
                    found, e->cap);
    }
    if (match && f.h_counts.p[2])
        return fail(err, errlen, OG_E_VERIFY,
                    "%u survivors' keys recomputed from their offsets differ from the search kernel's",
                    f.h_counts.p[2]);
    *count = match ? f.h_counts.p[1] : found;  // matches are at most the survivors
    *src = match ? (const void*)f.matches.p : (const void*)f.hits.p;
    return OG_OK;
}

// Copies n records of type Rec (HitRec or MatchRec, 48 bytes) from the
// device into h_recs on the copy stream, in up to COPY_CHUNKS chunks of at
// least 2^18 records, and runs body(lo, hi) over every record as soon as its
// chunk has arrived: the host threads convert one chunk while the next ones
// cross PCIe (config 3 returns 4e7 matches, 1.9 GB, an advance). Each of
// `workers` threads (host_workers(n) by default) takes its slice of every
// chunk. On an error every copy issued has ended before it returns.
template <class Rec, class F>
int copy_records(og_engine* e, const Rec* src, size_t n, F&& body, char* err, size_t errlen, size_t workers = 0) {
    static_assert(sizeof(Rec) == sizeof(HitRec), "the staging holds either record");
    if (n == 0) return OG_OK;
    Rec* const stage = reinterpret_cast<Rec*>(e->h_recs.p);
    constexpr size_t MIN_CHUNK = 1u << 18;
    const size_t chunks = std::min<size_t>(og_engine::COPY_CHUNKS, (n + MIN_CHUNK - 1) / MIN_CHUNK);
    const size_t per = (n + chunks - 1) / chunks;
    cudaError_t ce = cudaSuccess;
    for (size_t c = 0; c < chunks && ce == cudaSuccess; c++) {
        const size_t lo = c * per, hi = std::min(n, lo + per);
        ce = cudaMemcpyAsync(stage + lo, src + lo, (hi - lo) * sizeof(Rec), cudaMemcpyDeviceToHost, e->cstream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e->chunk_ev[c], e->cstream);
    }
    std::atomic<int> failed{(int)ce};
    const auto work = [&](size_t t, size_t nw) {
        for (size_t c = 0; c < chunks && failed.load() == cudaSuccess; c++) {
            const cudaError_t we = cudaEventSynchronize(e->chunk_ev[c]);
            if (we != cudaSuccess) {
                failed.store((int)we);
                return;
            }
            const size_t lo = c * per, hi = std::min(n, lo + per), slice = (hi - lo + nw - 1) / nw;
            const size_t a = std::min(hi, lo + t * slice), b = std::min(hi, a + slice);
            if (a < b) body(a, b);
        }
    };
    if (workers == 0) workers = host_workers(n);
    if (ce == cudaSuccess) {
        if (workers <= 1) {
            work(0, 1);
        } else {
            std::vector<std::thread> pool;
            for (size_t t = 0; t < workers; t++) pool.emplace_back([&work, t, workers] { work(t, workers); });
            for (std::thread& th : pool) th.join();
        }
    }
    if (failed.load() != cudaSuccess) {
        cudaStreamSynchronize(e->cstream);
        return fail(err, errlen, OG_E_DEVICE, "copying %zu records back: %s", n,
                    cuda_text((cudaError_t)failed.load()).c_str());
    }
    return OG_OK;
}
// With filters longer than the device tables reach, several can share the
// 12 symbols the device compared: the host's match (FilterSet::match_key)
// decides which, if any, each prefix record matches. Keeps the confirmed
// records, in order, at the front of `recs` and returns their count.
size_t confirm_matches(og_engine* e, MatchRec* recs, size_t n) {
    static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "limbs read as little-endian bytes");
    size_t k = 0;
    for (size_t j = 0; j < n; j++) {
        MatchRec m = recs[j];
        if (m.filter < e->prefix_count) {
            const long f = e->fs.match_key(reinterpret_cast<const uint8_t*>(m.y));
            if (f < 0) continue;
            m.filter = (uint32_t)f;
        }
        recs[k++] = m;
    }
    return k;
}

// The device writes matches in the caller's layout.
static_assert(sizeof(og_match) == sizeof(MatchRec) && offsetof(og_match, offset) == offsetof(MatchRec, offset) &&
                  offsetof(og_match, packed) == offsetof(MatchRec, y) &&
                  offsetof(og_match, filter) == offsetof(MatchRec, filter) &&
                  offsetof(og_match, pad) == offsetof(MatchRec, pad),
              "MatchRec is og_match's layout");
}  // namespace

extern "C" {

int og_device_count(int* count, char* err, size_t errlen) {
    if (!count) return fail(err, errlen, OG_E_ARG, "null argument");
    *count = 0;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorNoDevice || (e == cudaSuccess && n == 0))
        return fail(err, errlen, OG_E_NODEVICE, "the driver reports no device");
    if (e != cudaSuccess) return fail(err, errlen, OG_E_NODEVICE, "no usable CUDA driver (%s)", cuda_text(e).c_str());
    *count = n;
    return OG_OK;
}

int og_device_info(int ordinal, char* name, size_t namelen, uint64_t* memory, int* sms, char* err, size_t errlen) {
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, ordinal);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "device %d: %s", ordinal, cuda_text(e).c_str());
    if (name && namelen) snprintf(name, namelen, "%s", p.name);
    if (memory) *memory = p.totalGlobalMem;
    if (sms) *sms = p.multiProcessorCount;
    return OG_OK;
}

int og_engine_resident_lanes(int ordinal, uint32_t scheme, uint32_t block, uint32_t* lanes, char* err,
                             size_t errlen) {
    if (!lanes) return fail(err, errlen, OG_E_ARG, "null argument");
    if (scheme != OG_SCHEME_PAIRED && scheme != OG_SCHEME_CHAIN)
        return fail(err, errlen, OG_E_ARG, "unknown scheme %u", scheme);
    if (block == 0) block = 128;
    if (block % 32 != 0 || block > 1024) return fail(err, errlen, OG_E_ARG, "block %u: a multiple of 32 up to 1024", block);
    cudaError_t e = cudaSetDevice(ordinal);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "device %d: %s", ordinal, cuda_text(e).c_str());
    return resident_lanes(ordinal, scheme, 0, block, lanes, err, errlen);
}

int og_engine_new_config(int ordinal, const uint8_t start[128], const og_engine_config* cfg, const uint64_t* bitmap,
                         size_t words, uint32_t bits, og_engine** out, char* err, size_t errlen) {
    og_engine_config c{};
    if (cfg) c = *cfg;
    return build_engine(ordinal, start, c, bitmap, words, bits, out, err, errlen);
}

int og_engine_new_filters(int ordinal, const uint8_t start[128], const og_filters* f, const og_engine_config* cfg,
                          og_engine** out, char* err, size_t errlen) {
    if (!f || !out) return fail(err, errlen, OG_E_ARG, "null argument");
    og_engine_config c{};
    if (cfg) c = *cfg;
    og_engine* e = nullptr;
    int rc = build_engine(ordinal, start, c, nullptr, 0, 0, &e, err, errlen, f);
    if (rc != OG_OK) return rc;
    rc = enable_matching(e, f, err, errlen);
    if (rc != OG_OK) {
        og_engine_free(e);
        return rc;
    }
    *out = e;
    return OG_OK;
}

int og_engine_new(int ordinal, const uint8_t start[128], uint32_t threads, const uint64_t* bitmap, size_t words,
                  uint32_t bits, int retune, og_engine** out, char* err, size_t errlen) {
    og_engine_config cfg{};
    cfg.scheme = OG_SCHEME_PAIRED;
    if (threads != 0) {
        cfg.lanes = threads;
        return build_engine(ordinal, start, cfg, bitmap, words, bits, out, err, errlen);
    }
    char name[256] = "unnamed";
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, ordinal) == cudaSuccess) snprintf(name, sizeof name, "%s", p.name);
    const std::string key = device_key(name, "cuda", 0);
    Shape shape;
    if (!retune && tuning_get(key, shape) && shape.first && shape.second) {
        cfg.half = shape.first;
        cfg.lanes = shape.second;
        cfg.block = shape.block;
        cfg.rounds = shape.rounds;
        cfg.lanes_per_thread = shape.lanes_per_thread;
        if (build_engine(ordinal, start, cfg, bitmap, words, bits, out, err, errlen) == OG_OK) return OG_OK;
        // the remembered shape no longer builds: measure again
    }
    // Timed walk over lanes per thread, inversion batch and lanes in flight
    // (waves of the resident CTAs); the fastest is kept and recorded
    // (src/gpu/mod.rs:383-411; the reference's OpenCL tuner walks two
    // dimensions the same way, src/gpu/opencl.rs:207-271).
    og_engine* best = nullptr;
    double best_rate = -1;
    int last = OG_E_DEVICE;
    for (uint32_t lpt : {1u, 2u})
    for (uint32_t half : {512u, 1024u, 2048u}) {
        uint32_t resident = 0;
        if (resident_lanes(ordinal, OG_SCHEME_PAIRED, half, 128, &resident, err, errlen, lpt) != OG_OK) continue;
        for (uint32_t mult : {2u, 4u, 8u}) {
            og_engine_config c{};
            c.scheme = OG_SCHEME_PAIRED;
            c.half = half;
            c.lanes = resident * mult;
            c.block = 128;
            c.lanes_per_thread = lpt;
            og_engine* e = nullptr;
            last = build_engine(ordinal, start, c, bitmap, words, bits, &e, err, errlen);
            if (last != OG_OK) continue;
            std::vector<og_survivor> buf(og_engine_room(e));
            const double rate = time_advance(e, buf);
            if (rate > best_rate) {
                if (best) og_engine_free(best);
                best = e;
                best_rate = rate;
            } else {
                og_engine_free(e);
            }
        }
    }
    if (!best) return fail(err, errlen, last, "no launch shape this device would take");
    Shape s;
    s.first = best->cfg.half;
    s.second = best->cfg.lanes;
    s.block = best->cfg.block;
    s.rounds = best->cfg.rounds;
    s.lanes_per_thread = best->cfg.lanes_per_thread;
    s.rate = best_rate;
    s.at = unix_now();
    tuning_put(key, s);
    // hand back a fresh engine at the chosen shape: the timed one has moved on
    og_engine_config c = best->cfg;
    og_engine_free(best);
    return build_engine(ordinal, start, c, bitmap, words, bits, out, err, errlen);
}

uint32_t og_engine_threads(const og_engine* e) { return e ? e->cfg.lanes : 0; }

uint64_t og_engine_batch(const og_engine* e) {
    return e ? (uint64_t)e->cfg.lanes * e->slots * e->cfg.rounds : 0;
}

size_t og_engine_room(const og_engine* e) { return e ? e->cap : 0; }

void og_engine_shape(const og_engine* e, og_engine_config* cfg) {
    if (e && cfg) *cfg = e->cfg;
}

float og_engine_last_kernel_ms(const og_engine* e) { return e ? e->last_ms : 0.f; }

int og_engine_launch(og_engine* e, char* err, size_t errlen) { return enqueue_advance(e, false, err, errlen); }

int og_engine_collect(og_engine* e, og_survivor* out, size_t cap, size_t* n, char* err, size_t errlen) {
    if (!e || !n) return fail(err, errlen, OG_E_ARG, "null argument");
    *n = 0;
    uint32_t found = 0;
    uint64_t launch = 0;
    const void* src = nullptr;
    int rc = collect_flight(e, false, &found, &launch, &src, err, errlen);
    if (rc != OG_OK) return rc;
    if (found > cap) return fail(err, errlen, OG_E_CAPACITY, "%u survivors and room for %zu in the caller's buffer", found, cap);
    const uint64_t L = e->cfg.lanes, slots = e->slots, R = e->cfg.rounds;
    const bool paired = e->cfg.scheme == OG_SCHEME_PAIRED;
    static_assert(sizeof(og_survivor::packed) == sizeof(HitRec::y), "the packed key is the record's eight limbs");
    static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "limbs copied as little-endian bytes");
    rc = copy_records(e, static_cast<const HitRec*>(src), found, [&](size_t lo, size_t hi) {
        for (size_t k = lo; k < hi; k++) {
            const HitRec& h = e->h_recs.p[k];
            const uint64_t r = h.step / slots, i = h.step % slots;
            const uint64_t w = (launch * R + r) * L + h.lane;
            out[k].offset = paired ? 8 * (w * slots + 1 + i) : 8 * (w * slots + i);
            std::memcpy(out[k].packed, h.y, sizeof out[k].packed);
        }
    }, err, errlen);
    if (rc != OG_OK) return rc;
    *n = found;
    return OG_OK;
}

int og_engine_advance(og_engine* e, og_survivor* out, size_t cap, size_t* n, char* err, size_t errlen) {
    if (!e || !n) return fail(err, errlen, OG_E_ARG, "null argument");
    *n = 0;
    if (e->inflight) return fail(err, errlen, OG_E_STATE, "launched advances are not collected yet");
    const int rc = og_engine_launch(e, err, errlen);
    if (rc != OG_OK) return rc;
    return og_engine_collect(e, out, cap, n, err, errlen);
}

int og_engine_match_on_device(og_engine* e, const og_filters* f, char* err, size_t errlen) {
    if (!e || !f) return fail(err, errlen, OG_E_ARG, "null argument");
    if (e->cfg.dump) return fail(err, errlen, OG_E_STATE, "the engine keeps every candidate: it has no bitmap to match behind");
    if (f->has_suffixes && !e->sbitmap.p)
        return fail(err, errlen, OG_E_ARG,
                    "the filter set has suffixes and the engine no suffix bitmap: create it with og_engine_new_filters");
    if (!f->has_prefixes || f->set.bits() != e->bits)
        return fail(err, errlen, OG_E_ARG, "the filter set's index is %u bits wide and the engine's %u",
                    f->has_prefixes ? f->set.bits() : 0, e->bits);
    const size_t nwords = (size_t)(((1ULL << e->bits) + 63) / 64);
    if (f->set.words().size() < nwords || words_hash(f->set.words().data(), nwords) != e->bitmap_hash)
        return fail(err, errlen, OG_E_ARG, "the filter set's bitmap is not the one the engine was created with");
    return enable_matching(e, f, err, errlen);
}

int og_engine_launch_matches(og_engine* e, char* err, size_t errlen) {
    if (e && !e->matching) return fail(err, errlen, OG_E_STATE, "og_engine_match_on_device has not been called");
    return enqueue_advance(e, true, err, errlen);
}

int og_engine_collect_matches(og_engine* e, og_match* out, size_t cap, size_t* n, char* err, size_t errlen) {
    if (!e || !n) return fail(err, errlen, OG_E_ARG, "null argument");
    *n = 0;
    uint32_t matched = 0;
    uint64_t launch = 0;
    const void* src = nullptr;
    int rc = collect_flight(e, true, &matched, &launch, &src, err, errlen);
    if (rc != OG_OK) return rc;
    const MatchRec* dev = static_cast<const MatchRec*>(src);
    const MatchRec* stage = reinterpret_cast<const MatchRec*>(e->h_recs.p);
    if (!e->long_filters) {
        // every record is a match, already in the caller's layout: each
        // chunk is copied out as soon as it arrives
        if (matched > cap)
            return fail(err, errlen, OG_E_CAPACITY, "%u matches and room for %zu in the caller's buffer", matched, cap);
        rc = copy_records(e, dev, matched, [&](size_t lo, size_t hi) {
            std::memcpy(out + lo, stage + lo, (hi - lo) * sizeof(og_match));
        }, err, errlen);
        if (rc != OG_OK) return rc;
        *n = matched;
        return OG_OK;
    }
    rc = copy_records(e, dev, matched, [](size_t, size_t) {}, err, errlen, 1);
    if (rc != OG_OK) return rc;
    const size_t k = confirm_matches(e, reinterpret_cast<MatchRec*>(e->h_recs.p), matched);
    if (k > cap) return fail(err, errlen, OG_E_CAPACITY, "%zu matches and room for %zu in the caller's buffer", k, cap);
    std::memcpy(out, stage, k * sizeof(og_match));
    *n = k;
    return OG_OK;
}

int og_engine_collect_matches_view(og_engine* e, const og_match** matches, size_t* n, char* err, size_t errlen) {
    if (!e || !matches || !n) return fail(err, errlen, OG_E_ARG, "null argument");
    *matches = nullptr;
    *n = 0;
    uint32_t matched = 0;
    uint64_t launch = 0;
    const void* src = nullptr;
    int rc = collect_flight(e, true, &matched, &launch, &src, err, errlen);
    if (rc != OG_OK) return rc;
    // nothing to convert: the calling thread only waits for the chunks
    rc = copy_records(e, static_cast<const MatchRec*>(src), matched, [](size_t, size_t) {}, err, errlen, 1);
    if (rc != OG_OK) return rc;
    MatchRec* stage = reinterpret_cast<MatchRec*>(e->h_recs.p);
    *n = e->long_filters ? confirm_matches(e, stage, matched) : matched;
    *matches = reinterpret_cast<const og_match*>(stage);
    return OG_OK;
}

int og_engine_advance_matches(og_engine* e, og_match* out, size_t cap, size_t* n, char* err, size_t errlen) {
    if (!e || !n) return fail(err, errlen, OG_E_ARG, "null argument");
    *n = 0;
    if (e->inflight) return fail(err, errlen, OG_E_STATE, "launched advances are not collected yet");
    const int rc = og_engine_launch_matches(e, err, errlen);
    if (rc != OG_OK) return rc;
    return og_engine_collect_matches(e, out, cap, n, err, errlen);
}

void og_engine_free(og_engine* e) { delete e; }

}  // extern "C"
