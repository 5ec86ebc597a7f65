/*
 * CPU oracle for the onion-gen key-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a plain-C restatement of the
 * reference's CPU algorithms (onion-gen, Rust). Only the test suite, the
 * smoke check and the CPU-baseline leg of bench.py may load it, and only as
 * the checker or the timed CPU baseline. The product (libonion_gen_b200.so)
 * never links, loads or calls anything here.
 *
 * Every entry point names the reference function it restates. All byte
 * strings are little-endian; a "point" is four canonical 32-byte field
 * elements X, Y, Z, T (extended coordinates), 128 bytes in all.
 */
#ifndef ONION_ORACLE_H
#define ONION_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- field GF(2^255-19), src/field.rs ---------------------------------- */
void orc_fe_mul(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]);
void orc_fe_sq(const uint8_t a[32], uint8_t out[32]);
void orc_fe_add(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]);
void orc_fe_sub(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]);
void orc_fe_invert(const uint8_t a[32], uint8_t out[32]);
/* canonical encoding of an arbitrary value below 2^256 (Fe::to_bytes). */
void orc_fe_canon(const uint8_t a[32], uint8_t out[32]);

/* ---- group, src/curve.rs ------------------------------------------------- */
void orc_basepoint(uint8_t xyzt[128]);
void orc_scalar_base_mult(const uint8_t scalar[32], uint8_t xyzt[128]);
/* p + q for two points in extended coordinates (curve::add + to_p3). */
void orc_point_add(const uint8_t p[128], const uint8_t q[128], uint8_t out[128]);
/* k * 8G for a small k (pairs.rs multiple_of_eight_g). */
void orc_multiple_of_eight_g(uint64_t k, uint8_t xyzt[128]);
/* key::pack: y with the sign of x in bit 255. */
void orc_pack(const uint8_t xyzt[128], uint8_t out[32]);
/* affine x, y (canonical) of a point. */
void orc_to_affine(const uint8_t xyzt[128], uint8_t x[32], uint8_t y[32]);
/* 1 when L*B is the identity (curve.rs basepoint_has_expected_order). */
int orc_check_group_order(void);
/* 1 when the hard-coded 8G constant equals 3 doublings of B. */
int orc_check_eight_basepoint(void);

/* ---- hashes (FIPS 180-4 SHA-512, FIPS 202 SHA3-256) --------------------- */
void orc_sha512(const uint8_t *msg, size_t len, uint8_t out[64]);
void orc_sha3_256(const uint8_t *msg, size_t len, uint8_t out[32]);

/* ---- keys, src/key.rs ---------------------------------------------------- */
void orc_secret_scalar(const uint8_t seed[32], uint8_t sk[32]);
void orc_expanded_secret_key(const uint8_t seed[32], uint8_t out[64]);
/* returns 1 and fills out when clamping survives the offset, else 0. */
int orc_expanded_secret_at_offset(const uint8_t seed[32], uint64_t offset, uint8_t out[64]);
void orc_add_to_scalar(uint8_t sk[32], uint64_t delta);
int orc_clamping_intact(const uint8_t sk[32]);
void orc_public_key(const uint8_t seed[32], uint8_t out[32]);
void orc_checksum(const uint8_t pk[32], uint8_t out[2]);
/* 56 symbols + NUL. */
void orc_address(const uint8_t pk[32], char out[57]);
/* run.rs block_seed. */
void orc_block_seed(const uint8_t root[32], uint64_t index, uint8_t out[32]);

/* ---- base32, src/base32.rs ---------------------------------------------- */
/* writes ceil(8n/5) symbols + NUL; returns symbol count. */
size_t orc_base32_encode(const uint8_t *bytes, size_t n, char *out);
/* returns number of decoded bytes, or -(position+1) of the first bad symbol;
 * *bits receives 5*len. */
long orc_base32_decode_bits(const char *s, uint8_t *out, size_t cap, size_t *bits);

/* ---- engines -------------------------------------------------------------- */
/* BatchEngine (src/batch.rs:78-122): from `start`, runs batches of `batch`
 * until `count` candidates are produced; writes count*32 packed keys WITHOUT
 * the sign bit, element i = start scalar + 8i. `end` (nullable) receives the
 * accumulator after the last full batch. */
void orc_chain_keys(const uint8_t start[128], size_t batch, size_t count,
                    uint8_t *out, uint8_t end[128]);
/* the same keys WITH the sign bit (BatchEngine::packed_with_sign). */
void orc_chain_keys_signed(const uint8_t start[128], size_t batch, size_t count,
                           uint8_t *out);
/* chain keys over `threads` OS threads for big ranges: element i of the
 * output is start + 8*(first + i). */
void orc_chain_keys_mt(const uint8_t start[128], uint64_t first, size_t count,
                       uint8_t *out, int threads);
/* PairEngine (src/pairs.rs): begin() then `rounds` runs with no probe; for
 * every candidate writes its packed key (sign clear) and its delta. Output
 * order: round-major, candidate index ascending. */
void orc_pair_keys(const uint8_t start[128], size_t half, size_t rounds,
                   uint8_t *keys, uint64_t *deltas);
/* PairEngine::packed_with_sign for candidate `index` of the last round of a
 * fresh engine run for `rounds` rounds (deterministic re-run). */

/* Throughput of the paired engine (the product's default CPU engine,
 * src/run.rs:433-440) on `threads` threads for about `seconds` seconds after
 * one untimed round per thread (src/estimate.rs:86-117). Each thread starts
 * from its own seed. Returns candidates per second; *examined receives the
 * total counted. */
double orc_pair_rate(int threads, double seconds, size_t half, uint64_t *examined);
/* The same on one search: the scalar of `seed`, thread t starting 2^40 t
 * candidates into it (disjoint sub-ranges), every candidate probed in
 * `bitmap` (top `bits` bits of the packed key, src/filter.rs:2538-2549). */
double orc_pair_rate_search(int threads, double seconds, size_t half, const uint8_t seed[32], const uint64_t *bitmap,
                            uint32_t bits, uint64_t *examined);
/* Same for the chain engine (src/batch.rs). */
double orc_chain_rate(int threads, double seconds, size_t batch, uint64_t *examined);

/* ---- filters, src/filter.rs (literal prefixes only) --------------------- */
typedef struct orc_fset orc_fset;
/* newline-separated filters; bits == 0 chooses the width the way
 * FilterSet::new does (narrowest_acceptable). Returns NULL and a message on
 * a parse error or when no index can be built. */
orc_fset *orc_fset_new(const char *text, uint32_t bits, char *err, size_t errlen);
void orc_fset_free(orc_fset *s);
size_t orc_fset_count(const orc_fset *s);
/* canonical text of kept filter i (sorted, absorbed), NUL-terminated. */
void orc_fset_canonical(const orc_fset *s, size_t i, char *out, size_t cap);
uint32_t orc_fset_bits(const orc_fset *s);
size_t orc_fset_nwords(const orc_fset *s);
const uint64_t *orc_fset_words(const orc_fset *s);
double orc_fset_occupancy(const orc_fset *s);
int orc_fset_may_match(const orc_fset *s, const uint8_t packed[32]);
/* index of the first kept filter matching, or -1 (match_key). */
long orc_fset_match(const orc_fset *s, const uint8_t packed[32]);

/* ---- suffix filters, src/filter.rs (the `suffix:` form) ----------------- */
typedef struct orc_sset orc_sset;
/* newline-separated suffix bodies (without the "suffix:" form name): symbols,
 * `?` and `[...]` classes; bits == 0 chooses the width the way
 * FilterSet::with_index_bits does for suffixes. NULL and a message on a
 * parse error or when no suffix index can be built. */
orc_sset *orc_sset_new(const char *text, uint32_t bits, char *err, size_t errlen);
void orc_sset_free(orc_sset *s);
size_t orc_sset_count(const orc_sset *s);
uint32_t orc_sset_bits(const orc_sset *s);
size_t orc_sset_nwords(const orc_sset *s);
const uint64_t *orc_sset_words(const orc_sset *s);
/* the suffix index's bit test for a packed key (sign bit cleared). */
int orc_sset_may_match(const orc_sset *s, const uint8_t packed[32]);
/* Filter::key_prefilter of kept suffix i. */
int orc_sset_key_prefilter(const orc_sset *s, size_t i, const uint8_t packed[32]);
/* the first kept suffix the address of public key `pk` matches, or -1. */
long orc_sset_match_pk(const orc_sset *s, const uint8_t pk[32]);

/* ---- reference device bookkeeping --------------------------------------- */
/* src/gpu/cuda.rs:332-354: scalar offset of (tid, slot) in launch `launch`
 * for `threads` threads and HALF = half. */
uint64_t orc_cuda_offset(uint64_t tid, uint64_t slot, uint64_t launch,
                         uint32_t threads, uint32_t half);
/* src/gpu/mod.rs:306-312. */
uint32_t orc_hit_room(uint64_t batch, uint32_t bits);

#ifdef __cplusplus
}
#endif
#endif
