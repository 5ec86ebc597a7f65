/*
 * onion_gen_b200 — C ABI of the B200 key-search engine.
 *
 * A drop-in for the device engine onion-gen exposes to its run driver
 * (src/gpu/mod.rs:292-477, backend src/gpu/cuda.rs:103-365): a chain of
 * candidates starting at a point, filtered on the device by a prefix bitmap,
 * returning every (offset, packed key) the bitmap did not rule out.
 *
 * Conventions
 *   - Every call returns 0 (OG_OK) or an og_status; a message goes to
 *     `err` (NUL-terminated, truncated to `errlen`) when `err` is not NULL.
 *   - Field elements and keys are 32 little-endian bytes. A point is four
 *     field elements X, Y, Z, T (extended coordinates), 128 bytes.
 *   - An offset is the scalar delta of a candidate from the start point's
 *     scalar, always a multiple of 8 (src/gpu/mod.rs:113-119).
 *   - A packed key is the canonical y coordinate with the sign bit (bit 255)
 *     clear (src/gpu/mod.rs:117-118).
 *   - An engine is used by one thread at a time; distinct engines are
 *     independent.
 */
#ifndef ONION_GEN_B200_H
#define ONION_GEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum og_status {
    OG_OK = 0,
    OG_E_ARG = 1,        /* an argument is out of range */
    OG_E_NODEVICE = 2,   /* no driver or no device (src/gpu/cuda.rs:35-77) */
    OG_E_DEVICE = 3,     /* a CUDA call failed */
    OG_E_NOMEM = 4,      /* device or host memory could not be allocated */
    OG_E_OVERFLOW = 5,   /* more survivors than room: never truncated (src/gpu/cuda.rs:356-362) */
    OG_E_CAPACITY = 6,   /* the caller's output buffer is smaller than og_*_room() */
    OG_E_FILTER = 7,     /* a filter did not parse, or no index could be built */
    OG_E_STATE = 8,      /* call not valid in this state (unknown search, closed engine) */
    OG_E_TIMEOUT = 9,    /* a bounded wait ran out */
    OG_E_VERIFY = 10     /* an independent re-derivation disagreed with the device */
};

/* One candidate the bitmap did not rule out — gpu::Survivor
 * (src/gpu/mod.rs:113-119). */
typedef struct og_survivor {
    uint64_t offset;
    uint8_t packed[32];
} og_survivor;

/* ---- devices: cuda::look (src/gpu/cuda.rs:35-77) ----------------------- */

/* Number of CUDA devices; OG_E_NODEVICE when there is no driver or none. */
int og_device_count(int* count, char* err, size_t errlen);
/* Name and total memory of device `ordinal`. */
int og_device_info(int ordinal, char* name, size_t namelen, uint64_t* memory, int* sms, char* err,
                   size_t errlen);

/* ---- the engine: gpu::Engine (src/gpu/mod.rs:292-477) ------------------- */

typedef struct og_engine og_engine;

/* Replaces gpu::Engine::new(device, start, threads, bitmap, bitmap_bits,
 * retune) (src/gpu/mod.rs:346-413) and cuda::Engine::new
 * (src/gpu/cuda.rs:145-270). `start` is the chain's first point (s * B);
 * `threads` is the number of lanes, 0 to take the shape from tuning.yaml
 * or, failing that (or with `retune`), from a timed walk that is then
 * recorded there (src/tuning.rs). `bitmap` holds `words` 64-bit words of a
 * prefix index `bits` wide (FilterSet::index_words, src/filter.rs:1857). */
int og_engine_new(int ordinal, const uint8_t start[128], uint32_t threads, const uint64_t* bitmap,
                  size_t words, uint32_t bits, int retune, og_engine** out, char* err, size_t errlen);

/* Enumeration schemes. */
enum og_scheme {
    OG_SCHEME_PAIRED = 0, /* y(P +- Q_m) around an affine centre, one inversion per round */
    OG_SCHEME_CHAIN = 1   /* +8G chain, Z batch-inverted over n steps (src/batch.rs) */
};

/* Launch shape of an engine. Zero fields take defaults. */
typedef struct og_engine_config {
    uint32_t scheme;   /* og_scheme */
    uint32_t half;     /* paired: table size, a round is 2*half+1 candidates (0: 2048, halved
                          down to 256 while one advance would return more than 2^26 expected
                          survivors). chain: n steps (0: 1024) */
    uint32_t lanes;    /* lanes (independent chains), a multiple of `block`. The paired
                          kernel runs as many CTAs as are resident and they take the lanes
                          a block at a time, so its scratch is that of the resident CTAs
                          whatever the lanes (0: eight blocks per resident CTA, fewer only
                          if half 256 still passes that survivor budget). The chain kernel is
                          persistent the same way (0: four blocks per resident CTA) */
    uint32_t rounds;   /* rounds per advance */
    uint32_t block;    /* threads per CUDA block, a multiple of 32 */
    uint32_t dump;     /* 1: ignore the bitmap, every candidate survives (parity runs) */
    uint32_t room;     /* survivor records per advance; 0 sizes it from the bitmaps' occupancy:
                          the expected count plus eight standard deviations */
    uint32_t lanes_per_thread; /* paired: lanes each thread of the search kernel carries, 1 or 2
                          (0: 1); `lanes` is then a multiple of block x this. Chain: 1 */
} og_engine_config;

/* The same engine with an explicit shape (no tuning). `bitmap` may be NULL
 * only with cfg->dump = 1. */
int og_engine_new_config(int ordinal, const uint8_t start[128], const og_engine_config* cfg,
                         const uint64_t* bitmap, size_t words, uint32_t bits, og_engine** out, char* err,
                         size_t errlen);

/* Engine::threads (src/gpu/mod.rs:452): lanes. */
uint32_t og_engine_threads(const og_engine* e);
/* Engine::batch (src/gpu/mod.rs:461): candidates examined per advance. */
uint64_t og_engine_batch(const og_engine* e);
/* Survivor records one advance can return: the size `out` must have. */
size_t og_engine_room(const og_engine* e);
/* The shape in use. */
void og_engine_shape(const og_engine* e, og_engine_config* cfg);
/* Lanes one wave of the search kernel of `scheme` holds on device `ordinal`:
 * resident blocks per SM x SMs x `block` (0: 128). The paired kernel runs
 * exactly this many threads and they take the lanes a block at a time. */
int og_engine_resident_lanes(int ordinal, uint32_t scheme, uint32_t block, uint32_t* lanes, char* err,
                             size_t errlen);

/* Engine::advance (src/gpu/mod.rs:470, src/gpu/cuda.rs:282-365): moves every
 * lane on by one launch and writes each survivor to `out` (room `cap`),
 * their number to `*n`. More survivors than the engine's room is
 * OG_E_OVERFLOW, never a silent truncation. */
int og_engine_advance(og_engine* e, og_survivor* out, size_t cap, size_t* n, char* err, size_t errlen);

/* The same advance in two halves, so the host can work on one advance's
 * survivors while the next one runs: og_engine_launch enqueues an advance and
 * returns at once; og_engine_collect waits for the oldest launched advance
 * and returns its survivors (its records are copied on a stream of their
 * own, beside the next advance's kernel). At most two advances are in
 * flight (OG_E_STATE for a third launch, for a collect with none, and for
 * og_engine_advance while launches are pending). Results come back in launch
 * order and equal og_engine_advance's. */
int og_engine_launch(og_engine* e, char* err, size_t errlen);
int og_engine_collect(og_engine* e, og_survivor* out, size_t cap, size_t* n, char* err, size_t errlen);

/* Device time of the last collected advance's search kernel, milliseconds
 * (CUDA events on the engine's stream). */
float og_engine_last_kernel_ms(const og_engine* e);

/* ---- device-side exact match for the engine ------------------------------
 *
 * FilterSet::match_key (src/filter.rs:2194-2213, with the length buckets of
 * :2645-2700), which the reference runs on the host for every survivor
 * (run::device_worker, src/run.rs:1081-1085), moved onto the device: the
 * bitmap survivors of an advance are matched there and only exact matches
 * cross back. */

/* One exact match: the survivor and the index of the filter it matches in
 * the filter set's kept order (og_filters_text). */
typedef struct og_match {
    uint64_t offset;    /* scalar delta from the start, as og_survivor */
    uint8_t packed[32]; /* canonical y, sign bit cleared */
    uint32_t filter;
    uint32_t pad;
} og_match;

/* Turns the device match on. `f` must be the filter set whose index_words the
 * engine was created with (same width and the same bitmap, checked:
 * OG_E_ARG otherwise) and hold no suffix (an engine from og_engine_new has
 * no suffix bitmap); its exact-match tables are copied and `f` is not
 * referenced afterwards. An engine created with dump = 1 has no bitmap and
 * refuses (OG_E_STATE). */
int og_engine_match_on_device(og_engine* e, const struct og_filters* f, char* err, size_t errlen);

/* An engine over a whole filter set, prefixes and suffixes (shape as
 * og_engine_new_config; dump must be 0), with the device match already on.
 * Candidates survive the kernel through the prefix bitmap or the suffix
 * bitmap (og_filters_suffix_words); a suffix survivor's key is recomputed
 * on the device from its offset, sign bit and SHA3-256 checksum included
 * (src/key.rs:106-132), and matched on its address. Suffix matches carry
 * filter index og_filters_prefix_count(f) + j. */
int og_engine_new_filters(int ordinal, const uint8_t start[128], const struct og_filters* f,
                          const og_engine_config* cfg, og_engine** out, char* err, size_t errlen);

/* One advance that returns only the exact matches (room `cap`, count `*n`).
 * Survivors beyond the engine's room are OG_E_OVERFLOW as in
 * og_engine_advance; a recomputed suffix key that differs from the search
 * kernel's is OG_E_VERIFY. Filters longer than 12 symbols are matched on their
 * first 12 on the device and confirmed on the host before they are
 * returned. */
int og_engine_advance_matches(og_engine* e, og_match* out, size_t cap, size_t* n, char* err, size_t errlen);
/* og_engine_advance_matches in two halves, as og_engine_launch /
 * og_engine_collect. */
int og_engine_launch_matches(og_engine* e, char* err, size_t errlen);
int og_engine_collect_matches(og_engine* e, og_match* out, size_t cap, size_t* n, char* err, size_t errlen);
/* og_engine_collect_matches without the copy into the caller's buffer: the
 * oldest advance's `*n` matches are left in the engine's own pinned host
 * memory, which the device writes into directly, and `*matches` points at
 * them. They stay valid until the next collect of any kind or
 * og_engine_free; a caller that keeps them copies them first. The same
 * errors as og_engine_collect_matches, bar OG_E_CAPACITY (the engine's room
 * holds every match). */
int og_engine_collect_matches_view(og_engine* e, const og_match** matches, size_t* n, char* err, size_t errlen);

void og_engine_free(og_engine* e);

/* ---- the batched engine: many searches in one persistent kernel ---------
 *
 * No counterpart in the reference (its device engine runs one search per
 * device thread, src/run.rs:1030-1119). Every search is a seeded base scalar
 * (key::secret_scalar, src/key.rs:23-29), a literal-prefix filter set and a
 * quota. All admitted searches advance together: one step replays a captured
 * CUDA graph that runs one persistent kernel over every search's lanes, then
 * matches the bitmap survivors exactly on the device. Every exact hit is
 * re-derived and verified on the host before it counts (src/run.rs:1089-1111).
 *
 * A search's result is its first `quota` hits in offset order. Offsets are a
 * pure function of the search (candidate windows are processed in contiguous
 * increasing order whatever the lanes it holds), so the result is the same
 * whether the search runs alone or beside any others. */

typedef struct og_batch og_batch;

typedef struct og_batch_config {
    uint32_t half;          /* table size of every search; a round is 2*half+1 keys (0: 256) */
    uint32_t slots;         /* lanes in the shared pool, a multiple of 128 (0: two waves of resident blocks) */
    uint32_t rounds;        /* rounds per step (0: 1) */
    uint32_t max_searches;  /* searches admitted at once (0: 4096) */
    uint32_t max_hits;      /* exact hits one step may return (0: 65536) */
    uint32_t graph;         /* 0 or 1: replay each step as a captured CUDA graph; 2: plain launches */
    uint32_t grid;          /* persistent CTAs per SM (0: as many as fit) */
    uint64_t memory_budget; /* device bytes for per-search tables (0: half of the free memory after the pool) */
    uint32_t max_half;      /* largest inversion batch a search may run at (0: `half`): a search runs at
                               half doubled while its expected work (quota over its filters' match
                               probability) covers at least four steps of the whole pool at the doubled
                               half; a power-of-two multiple of `half`, at most 2048 */
    uint32_t inflight;      /* steps queued on the device at once, 1 or 2 (0: 2): og_batch_step
                               launches the next step before it collects the oldest, so the host's
                               work on one step's hits overlaps the next step */
} og_batch_config;

typedef struct og_batch_hit {
    uint64_t search_id;
    uint64_t offset;     /* scalar delta from the search's base scalar */
    uint8_t packed[32];  /* the public key, sign bit clear */
    uint8_t public_key[32]; /* the full public key (sign set), as re-derived on the host */
    uint32_t filter;     /* index of the matching filter in the search's sorted set */
    uint32_t pad;
} og_batch_hit;

typedef struct og_search_status {
    uint64_t windows;    /* candidate windows fully processed */
    uint64_t candidates; /* = windows * (2*half+1) */
    uint64_t hits;       /* verified hits found so far */
    uint32_t lanes;      /* lanes held in the last step */
    uint32_t quota;
    uint32_t done;       /* 1 once the first `quota` hits are known */
    uint32_t filters;
    uint64_t table_bytes;/* device bytes of its bitmap and exact-match tables */
    uint32_t status;     /* OG_OK, or OG_E_VERIFY when one of its device hits did not re-derive on
                            the host (it is then done, with the hits verified before) */
    uint32_t half;       /* its inversion batch */
} og_search_status;

int og_batch_new(int ordinal, const og_batch_config* cfg, og_batch** out, char* err, size_t errlen);

/* The batch's autotuner. Times a synthetic mix of `searches` searches (0:
 * 64) that never reach their quota at every shape of inversion batch (half
 * 128, 256, 512), slot pool (1, 2, 3 waves of persistent CTAs) and grid
 * (all resident CTAs per SM, or half of them), keeps the highest keys/s
 * whose step stays within `max_step_ms` of device time (0: no cap),
 * records it in tuning.yaml under `device/<name>/cuda-batch/0/<version>`
 * (first = half, second = slots, block = grid, rounds) and writes it to
 * `out` (other fields zero: defaults). og_batch_new takes the recorded
 * shape when half, slots, rounds and grid are all 0. */
int og_batch_tune(int ordinal, uint32_t searches, float max_step_ms, og_batch_config* out, double* keys_per_s,
                  char* err, size_t errlen);
/* The shape a batch runs (defaults filled in). */
void og_batch_shape(const og_batch* b, og_batch_config* cfg);
/* Admits a search: `filters` newline-separated, literal prefixes and
 * `suffix:` lines as og_filters_new takes them (a suffix hit's key, sign
 * bit and checksum are recomputed on the device). Fails with OG_E_NOMEM
 * when its tables do not fit the memory budget (nothing is changed),
 * OG_E_CAPACITY when max_searches are admitted, OG_E_FILTER when its
 * bitmaps would let more than 2% of the candidates through. */
int og_batch_admit(og_batch* b, uint64_t search_id, const uint8_t seed[32], const char* filters, uint32_t quota,
                   char* err, size_t errlen);
/* One step: every admitted, unfinished search advances `rounds` rounds.
 * With `inflight` 2 the call first launches the next step (so that up to two
 * are queued on the device), then waits for the oldest and writes its
 * verified hits to `out` (room `cap`; `out` NULL: none are copied, they stay
 * in og_batch_results); a search whose quota
 * the oldest step meets may still hold lanes in the newer one, and the device
 * skips them. Errors:
 *   OG_E_VERIFY   a device hit of some searches did not re-derive on the host:
 *                 those searches end (og_search_status.status), the other
 *                 searches' hits of the step are in `out`, and the batch goes on;
 *   OG_E_OVERFLOW a step's survivors or hits exceeded their room: the batch
 *                 closes, and every later call fails with OG_E_STATE;
 *   OG_E_DEVICE   a CUDA call failed: the batch closes likewise. */
int og_batch_step(og_batch* b, og_batch_hit* out, size_t cap, size_t* n, char* err, size_t errlen);
size_t og_batch_room(const og_batch* b);
int og_batch_status(const og_batch* b, uint64_t search_id, og_search_status* st);
/* The result of a finished search: its first `quota` hits in offset order. */
int og_batch_results(const og_batch* b, uint64_t search_id, og_batch_hit* out, size_t cap, size_t* n);
/* Removes a search (finished or not) and frees its lanes and tables. The
 * tables go back to the batch's pool in stream order, after the steps
 * already launched: the call does not wait for the device. */
int og_batch_retire(og_batch* b, uint64_t search_id);
/* Searches admitted and not yet retired; of them, unfinished. */
void og_batch_counts(const og_batch* b, size_t* admitted, size_t* running);
/* Device time of the last step (CUDA events around the graph), ms. */
float og_batch_last_step_ms(const og_batch* b);
/* Candidates examined in the last step, all searches. */
uint64_t og_batch_last_step_candidates(const og_batch* b);
/* Kernel launches the last step made (graph nodes that are kernels). */
uint32_t og_batch_last_step_launches(const og_batch* b);
/* Device bytes of per-search tables in use, and the budget. */
void og_batch_memory(const og_batch* b, uint64_t* used, uint64_t* budget);
/* For tests of the failure path: the host treats the next hit of the search
 * that it verifies as one that did not re-derive. The fault is made on the
 * host; nothing on the device changes. */
int og_batch_plant_mismatch(og_batch* b, uint64_t search_id);
void og_batch_free(og_batch* b);

/* ---- serving: a request loop over the batched engine -------------------
 *
 * No counterpart in the reference. A worker thread owns one og_batch and
 * runs steps continuously. Requests submitted from any thread wait in a FIFO
 * queue and are admitted as lanes and device memory allow (a request the
 * memory budget cannot take yet stays queued; one that can never parse
 * completes with an error status). Each step advances every admitted request
 * together; a request completes, and is retired, at the end of the step in
 * which its quota of verified hits is reached. Its result is the same as if
 * it had run alone (the batched engine's guarantee). Times are
 * CLOCK_MONOTONIC nanoseconds. */

typedef struct og_serve og_serve;

typedef struct og_serve_config {
    og_batch_config batch;  /* the engine the loop drives */
    uint32_t max_running;   /* requests admitted at once (0: the batch's max_searches) */
    uint32_t reserved;
} og_serve_config;

typedef struct og_serve_done {
    uint64_t request_id;
    uint64_t arrival_ns;   /* when og_serve_submit accepted it */
    uint64_t admit_ns;     /* when it got a place on the device */
    uint64_t done_ns;      /* end of the step that completed it */
    uint64_t candidates;   /* candidates it examined */
    uint32_t hits;         /* verified hits returned (its quota unless status != 0) */
    uint32_t status;       /* og_status: OG_OK, or why it could not run */
} og_serve_done;

typedef struct og_serve_stats {
    uint64_t steps;
    uint64_t candidates;   /* all requests, all steps */
    double device_ms;      /* sum of step device times */
    uint64_t queued;       /* waiting for admission */
    uint64_t running;      /* admitted, unfinished */
    uint64_t completed;
} og_serve_stats;

int og_serve_new(int ordinal, const og_serve_config* cfg, og_serve** out, char* err, size_t errlen);
/* Queues a request (thread-safe); the arrival time is taken here. `filters`
 * as og_batch_admit takes them; a request the batch refuses completes with
 * that status. */
int og_serve_submit(og_serve* s, uint64_t request_id, const uint8_t seed[32], const char* filters, uint32_t quota,
                    char* err, size_t errlen);
/* Requests completed since the last poll, in completion order. */
int og_serve_poll(og_serve* s, og_serve_done* out, size_t cap, size_t* n);
/* The hits of a completed request (its first `quota` in offset order); they
 * are kept until fetched once. */
int og_serve_results(og_serve* s, uint64_t request_id, og_batch_hit* out, size_t cap, size_t* n);
void og_serve_stats_get(og_serve* s, og_serve_stats* st);
/* Nanoseconds on the clock the loop stamps with. */
uint64_t og_serve_now_ns(void);
/* Stops the loop (after its current step) and frees everything. */
void og_serve_free(og_serve* s);

/* ---- a search that allocates nothing ------------------------------------
 *
 * No counterpart in the reference. For callers that cannot allocate device
 * memory — code inside another framework's memory pool, callers that must not
 * synchronise the device (cudaMalloc and cudaFree can), processes that
 * reserve all device memory up front — og_search_noalloc runs one paired
 * search over a fixed range without calling cudaMalloc, cudaFree or any
 * allocating library routine. The caller passes the inputs and outputs in
 * device memory it owns; lane state, the Montgomery scratch and the tables
 * live in one file-scope device array of OG_NOALLOC_SCRATCH_BYTES, which
 * every GPU that loads this library holds until the process exits.
 *
 * It examines the first lanes * rounds * (2 half + 1) candidates of `start`
 * (offsets 8 .. 8 N), exactly as og_engine_advance does on a fresh engine
 * of the same shape, and writes each bitmap survivor (every candidate when
 * `d_bitmap` is NULL) to `d_hits` (room `cap`) and their number to
 * `*d_count` (zeroed by the call; a count above `cap` means records were
 * dropped). A record's offset is 8 (w (2 half + 1) + 1 + i) with
 * w = (step / (2 half + 1)) * lanes + lane and i = step % (2 half + 1).
 *
 * Limits: lanes a multiple of 128, half <= 2048, and
 * lanes * (2 half + 3) * 64 + half * 96 <= OG_NOALLOC_SCRATCH_BYTES;
 * beyond that the call fails with OG_E_CAPACITY before touching the device.
 * Work is enqueued on `stream` (a cudaStream_t; NULL for the legacy default
 * stream) and the call returns without waiting for it: it enqueues one
 * memset of `*d_count` and three kernels, whose constants travel as launch
 * parameters, and copies nothing from host memory.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call shares the one array: calls whose work overlaps on the GPU
 * (different streams or host threads without ordering) race. */
#define OG_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)

typedef struct og_hit_record {
    uint32_t lane;
    uint32_t step;
    uint32_t search;
    uint32_t reserved;
    uint32_t y[8]; /* the packed key's little-endian words, sign bit clear */
} og_hit_record;

int og_search_noalloc(int ordinal, const uint8_t start[128], uint32_t lanes, uint32_t half, uint32_t rounds,
                      const uint32_t* d_bitmap, uint32_t bits, og_hit_record* d_hits, uint32_t cap, uint32_t* d_count,
                      void* stream, char* err, size_t errlen);

/* ---- measurement --------------------------------------------------------- */

/* The integer-multiply roofline of device `ordinal`, measured: the issue
 * rate of independent 32-bit multiply-adds (per second) and the partial
 * products per second that independent field multiplications achieve.
 * No counterpart in the reference (its engine reports candidates/s only). */
int og_measure_int_peak(int ordinal, double* imad_per_s, double* mul_pp_per_s, char* err, size_t errlen);

/* ---- host side of the hit path ------------------------------------------ */

/* key::secret_scalar (src/key.rs:23-29). */
void og_secret_scalar(const uint8_t seed[32], uint8_t scalar[32]);
/* key::expanded_secret_key (src/key.rs:33-39). */
void og_expanded_secret_key(const uint8_t seed[32], uint8_t out[64]);
/* key::expanded_secret_at_offset (src/key.rs:167-177): 0 when clamping broke. */
int og_expanded_secret_at_offset(const uint8_t seed[32], uint64_t offset, uint8_t out[64]);
/* curve::scalar_base_mult (src/curve.rs:188-198), point as X,Y,Z,T. */
void og_scalar_base_mult(const uint8_t scalar[32], uint8_t point[128]);
/* key::pack (src/key.rs:55-62). */
void og_pack(const uint8_t point[128], uint8_t out[32]);
/* key::address (src/key.rs:118-132), 56 symbols + NUL. */
void og_address(const uint8_t pk[32], char out[57]);
/* run::block_seed (src/run.rs:211-221). */
void og_block_seed(const uint8_t root[32], uint64_t index, uint8_t out[32]);
/* The device-key recheck of src/run.rs:1089-1104: re-derives the candidate
 * at `offset` from `seed` and compares it with `packed` (sign masked).
 * OG_OK fills the full public key and the 64-byte secret; OG_E_VERIFY on a
 * mismatch; OG_E_ARG when the offset broke clamping. */
int og_check_hit(const uint8_t seed[32], uint64_t offset, const uint8_t packed[32], uint8_t pk[32],
                 uint8_t secret[64]);

/* ---- filters: FilterSet (src/filter.rs) -------------------------------- */

typedef struct og_filters og_filters;

/* Newline-separated filters (Pattern::parse, src/filter.rs:298-350):
 * prefixes (bare, `^` or `prefix:`) and `suffix:` forms, whose symbols may
 * be `?` or `[...]` classes (parse_symbols, :495-560); suffixes are checked
 * against the v3 address tail (:566-600). A prefix with wildcards or classes
 * fills every slot it allows in the prefix bitmap (pattern_slots,
 * :2480-2530; more than 4096 slots cannot be indexed: OG_E_FILTER) and is
 * matched after the literal prefixes, in order. `bits` is the prefix index width, 0 to choose
 * it; the suffix index width is always chosen (:1420-1440). A suffix that
 * reaches too little of the key for a suffix bitmap is OG_E_FILTER. */
int og_filters_new(const char* text, uint32_t bits, og_filters** out, char* err, size_t errlen);
/* Kept filters: the prefixes (sorted, absorbed) first, then the suffixes
 * (sorted, duplicates dropped). */
size_t og_filters_count(const og_filters* f);
size_t og_filters_prefix_count(const og_filters* f);
/* canonical text of kept filter i ("suffix:..." for a suffix) */
int og_filters_text(const og_filters* f, size_t i, char* out, size_t cap);
/* The prefix index (FilterSet::index_words, src/filter.rs:1857); 0 words
 * when the set has no prefix. */
uint32_t og_filters_bits(const og_filters* f);
size_t og_filters_words(const og_filters* f, const uint64_t** words);
/* The suffix index (BitmapIndex::build_over_suffixes, src/filter.rs:2406):
 * keyed on base32 bits [255 - bits, 255) of the packed key; 0 words when the
 * set has no suffix. */
uint32_t og_filters_suffix_bits(const og_filters* f);
size_t og_filters_suffix_words(const og_filters* f, const uint64_t** words);
/* The full check of a public key (sign bit included) against every filter,
 * on its address (FilterSet::match_address, src/filter.rs:2152): the index
 * of the first match or -1. */
long og_filters_match_address(const og_filters* f, const uint8_t pk[32]);
double og_filters_occupancy(const og_filters* f);
/* FilterSet::probability (src/filter.rs:1979-1990): the chance that a
 * uniform key's address matches some filter, 1 - prod(1 - p_f) over the kept
 * filters, each p_f the product over its symbols of the accepted symbols the
 * v3 protocol can produce there over those it can (src/filter.rs:226-238,
 * 443-452). The expected candidates to a hit are its inverse
 * (src/estimate.rs:69-78). */
double og_filters_match_probability(const og_filters* f);
/* FilterSet::match_key (src/filter.rs:2098): index of the match or -1. */
long og_filters_match(const og_filters* f, const uint8_t packed[32]);
/* match_key over `n` keys laid out `stride` bytes apart (a survivor array's
 * packed fields): writes each key's match or -1 to `out`, returns the number
 * that matched. */
size_t og_filters_match_many(const og_filters* f, const uint8_t* packed, size_t n, size_t stride, int32_t* out);
void og_filters_free(og_filters* f);

#ifdef __cplusplus
}
#endif
#endif
