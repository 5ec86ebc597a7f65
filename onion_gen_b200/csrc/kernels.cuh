// Device kernels of the key search and the host-side launch interface.
//
// Two enumeration schemes share one back end (Montgomery batch inversion,
// canonical packing, prefix-bitmap test, warp-aggregated hit append):
//
//  * paired (the production engine). A lane holds an affine centre P. One
//    round yields y(P + Q_m) and y(P - Q_m) for the table Q_m = 8m G,
//    m = 1..half, plus y(P) itself, from the dedicated Edwards formulas
//        y(P + Q) = (t1 - t2) / (x1 y2 - y1 x2),
//        y(P - Q) = (t1 + t2) / (x1 y2 + y1 x2),      t = x y,
//    i.e. two multiplications per pair, and moves P to the next centre
//    P + W with x(P + W) = (t1 + tW) / (y1 yW - x1 xW) whose two divisions
//    ride in the same batch. Every denominator of the round is inverted with
//    one field inversion (Montgomery's trick, numerators folded into the
//    forward products as in src/pairs.rs:174-224).
//  * chain (the contract of src/batch.rs): a lane steps its projective point
//    by +8G (seven multiplications, the addend's Z scaled to one) and
//    batch-inverts Z over its `n` steps.
//
// Candidate numbering. Lane l of L in global round r ("window" w = r L + l):
//   paired: index i in [0, 2 half] is the key of scalar offset
//           8 (w (2 half + 1) + 1 + i); i = half is the centre, i = half + m
//           is P + Q_m, i = half - m is P - Q_m.
//   chain:  index t in [0, n) is the key of scalar offset 8 (w n + t).
// Offsets never collide across lanes or rounds, and a run of R rounds covers
// every candidate index of its range exactly once.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace og {

// One bitmap survivor: 48 bytes, three 16-byte stores.
struct HitRec {
    uint32_t lane;
    uint32_t step;  // round-in-launch * slots + candidate index
    uint32_t search;
    uint32_t pad;
    uint32_t y[8];  // canonical y, little-endian limbs (the packed key, sign bit clear)
};
static_assert(sizeof(HitRec) == 48, "HitRec layout");

// A device exact match in the caller's layout (og_match): the candidate's
// scalar offset, its canonical y limbs (the packed key's little-endian
// bytes) and the filter it matched. The match kernel decodes the offset, so
// the host copies the records through unchanged.
struct MatchRec {
    uint64_t offset;
    uint32_t y[8];
    uint32_t filter;
    uint32_t pad;
};
static_assert(sizeof(MatchRec) == 48, "MatchRec layout");

struct FeWords {
    uint32_t v[8];
};

struct PairedArgs {
    const uint4* table;      // Q_m, m = 1..half: ((m-1)*3 + {x,y,t}) * 2 + q
    uint4* lanes;            // affine centres: ({x,y} * 2 + q) * L + lane
    uint4* scratch;          // ((e * 2 + {num,den}) * 2 + q) * S + slot, e < 2 half + 2
    uint32_t* work;          // next block of lanes to take, zero at launch
    uint32_t slots_n;        // S: persistent CTAs x block, the scratch slots
    const uint32_t* bitmap;  // prefix bitmap as 32-bit words (nullptr: none)
    uint32_t bits;
    HitRec* hits;
    uint32_t* counter;
    uint32_t cap;
    uint32_t search;         // copied into every record
    const uint32_t* sbitmap; // suffix bitmap (nullptr: none); with neither bitmap every candidate survives
    uint32_t sbits;
    FeWords wx, wy, wt;      // the round stride W = L (2 half + 1) 8 G, affine
    uint32_t lanes_n;        // L, a multiple of the block size times lanes_per_thread
    uint32_t half;
    uint32_t rounds;         // rounds per launch
    uint32_t lanes_per_thread;  // 1 (paired_kernel) or 2 (paired_kernel2); S = CTAs x block x this
    uint32_t stage_records;  // 1: survivors staged per warp in shared memory (one lane a thread only)
};

// Rows of a chain CTA's scratch hold this many threads (the largest block).
constexpr uint32_t CHAIN_ROW = 128;

struct ChainArgs {
    uint4* lanes;            // projective points: ({X,Y,Z,T} * 2 + q) * L + lane
    // per persistent CTA c a region of CHAIN_ROW * 4 n uint4 from c CHAIN_ROW 4 n:
    // thread j's step t, part w ({num,den}), half q at ((t * 2 + w) * 2 + q) CHAIN_ROW + j
    uint4* scratch;
    uint32_t* work;          // blocks of lanes taken so far this launch (starts at 0)
    uint32_t slots_n;        // persistent CTAs x block
    const uint32_t* bitmap;
    uint32_t bits;
    HitRec* hits;
    uint32_t* counter;
    uint32_t cap;
    uint32_t search;
    const uint32_t* sbitmap;
    uint32_t sbits;
    FeWords step_ypx, step_ymx, step_t2d;  // +8G, Z = 1
    FeWords jump_ypx, jump_ymx, jump_t2d;  // +8 (L-1) n G, Z = 1 (unused when L = 1)
    uint32_t lanes_n;
    uint32_t n;
    uint32_t rounds;
};

// Lane start points: lane l starts at base + l * stride, built from the
// binary expansion of l over `pow2` = { 2^k stride } in cached form with
// Z = 1 (y+x, y-x, 2dxy). `affine_out` selects the paired layout (x, y)
// over the chain layout (X, Y, Z, T).
struct InitArgs {
    uint4* lanes;
    FeWords bx, by, bz, bt;  // base point, extended
    const uint4* pow2;       // (k * 3 + {ypx,ymx,t2d}) * 2 + q
    uint32_t nbits;
    uint32_t lanes_n;
    uint32_t affine_out;
};

// Exact-match tables of a literal-prefix filter set in the form the device
// searches (FilterSet::match_key, src/filter.rs:2194-2213, with the length
// buckets of :2645-2700): one bucket per distinct filter length of at most
// 12 symbols, each a sorted run of masked 64-bit key heads (bytes 0..7 of the
// packed key, big-endian) with the owning filter's index.
constexpr int MAX_MATCH_BUCKETS = 12;
struct MatchTables {
    const uint64_t* keys;
    const uint32_t* owners;
    uint32_t nbuckets;
    uint32_t bucket_bits[MAX_MATCH_BUCKETS];
    uint32_t bucket_off[MAX_MATCH_BUCKETS];
    uint32_t bucket_len[MAX_MATCH_BUCKETS];
    // prefixes with wildcards or classes, walked after the buckets: per
    // pattern PATTERN_WORDS words, its filter index, the key-only symbols it
    // fixes (at most 49) and one symbol set per position
    const uint32_t* patterns;
    uint32_t npatterns;
};
constexpr uint32_t PATTERN_WORDS = 2 + 49;

// The single engine's exact match over one advance's bitmap survivors:
// matching records are copied to `out` with `pad` = the filter's index.
// Prefixes are matched on the key (MatchTables). A survivor whose slot is
// set in the suffix bitmap has its full key recomputed from its offset
// (start + k 8G), sign bit and checksum included, and is matched on its
// address against every suffix.
constexpr uint32_t MAX_SUFFIX_SYMBOLS = 56;
struct MatchArgs {
    const HitRec* surv;
    const uint32_t* surv_count;
    uint32_t surv_cap;
    MatchTables t;           // nbuckets = 0: no prefixes
    const uint32_t* sbitmap; // suffix bitmap, nullptr: no suffixes
    uint32_t sbits;
    const uint32_t* suffixes;  // per suffix 57 words: its length, then one symbol set per position
    uint32_t nsuffix;
    uint32_t prefix_count;     // filter index of suffix j is prefix_count + j
    FeWords sx, sy, sz, st;    // the engine's start point, extended
    const uint4* pow8;         // 2^j 8G, j < 64, cached form: (j * 3 + {ypx,ymx,t2d}) * 2 + q
    uint64_t window0;          // first window of the advance: launch * rounds * lanes
    uint32_t lanes;
    uint32_t slots;
    uint32_t paired;           // offsets 8 (w slots + 1 + i), else 8 (w slots + i)
    MatchRec* out;
    uint32_t* out_count;
    uint32_t out_cap;
    uint32_t* mismatch;        // survivors whose recomputed key differs from their record
};

cudaError_t launch_init(const InitArgs& a, int block, cudaStream_t s);
cudaError_t launch_match(const MatchArgs& a, int grid, cudaStream_t s);
// The paired kernel is persistent: `grid` CTAs (the resident ones) take the
// lanes a block at a time (two blocks with two lanes per thread) from
// `work`, so the scratch covers only the lanes in flight and no SM idles in
// a tail wave.
cudaError_t launch_paired(const PairedArgs& a, int block, int grid, cudaStream_t s);
cudaError_t launch_chain(const ChainArgs& a, int block, int grid, cudaStream_t s);

// Register and shared-memory footprint of the search kernels, for the shape
// choice.
struct KernelInfo {
    int regs;
    int max_threads;
    size_t local_bytes;
    int blocks_per_sm;
};
cudaError_t paired_info(int block, uint32_t half, uint32_t lanes_per_thread, KernelInfo* info);
cudaError_t chain_info(int block, KernelInfo* info);

}  // namespace og
