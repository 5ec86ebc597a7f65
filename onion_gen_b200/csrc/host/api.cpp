// C ABI of the host side of the hit path: keys, re-derivation, filters.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../../include/onion_gen_b200.h"
#include "common.h"
#include "filters.h"
#include "keys.h"

using namespace og;

extern "C" {

void og_secret_scalar(const uint8_t seed[32], uint8_t scalar[32]) { secret_scalar(seed, scalar); }

void og_expanded_secret_key(const uint8_t seed[32], uint8_t out[64]) { expanded_secret_key(seed, out); }

int og_expanded_secret_at_offset(const uint8_t seed[32], uint64_t offset, uint8_t out[64]) {
    return expanded_secret_at_offset(seed, offset, out) ? 1 : 0;
}

void og_scalar_base_mult(const uint8_t scalar[32], uint8_t point[128]) { point_to_bytes(base_mult(scalar), point); }

void og_pack(const uint8_t point[128], uint8_t out[32]) { pt_encode(point_from_bytes(point), out); }

void og_address(const uint8_t pk[32], char out[57]) {
    const std::string a = address(pk);
    std::memcpy(out, a.c_str(), 57);
}

void og_block_seed(const uint8_t root[32], uint64_t index, uint8_t out[32]) { block_seed(root, index, out); }

int og_check_hit(const uint8_t seed[32], uint64_t offset, const uint8_t packed[32], uint8_t pk[32], uint8_t secret[64]) {
    uint8_t p[32], s[64];
    switch (check_hit(seed, offset, packed, p, s)) {
        case HitCheck::ok:
            if (pk) std::memcpy(pk, p, 32);
            if (secret) std::memcpy(secret, s, 64);
            return OG_OK;
        case HitCheck::clamping:
            return OG_E_ARG;
        default:
            return OG_E_VERIFY;
    }
}

int og_filters_new(const char* text, uint32_t bits, og_filters** out, char* err, size_t errlen) {
    if (!text || !out) return fail(err, errlen, OG_E_ARG, "null argument");
    *out = nullptr;
    std::vector<PrefixFilter> fs;
    std::vector<SuffixPattern> sfx;
    std::string perr;
    if (!parse_filter_lines(text, fs, sfx, perr)) return fail(err, errlen, OG_E_FILTER, "%s", perr.c_str());
    if (fs.empty() && sfx.empty()) return fail(err, errlen, OG_E_FILTER, "no filters");
    og_filters* h = new (std::nothrow) og_filters();
    if (!h) return fail(err, errlen, OG_E_NOMEM, "host memory");
    std::string why;
    if (!fs.empty()) {
        if (!h->set.build(std::move(fs), bits, why)) {
            delete h;
            return fail(err, errlen, OG_E_FILTER, "%s", why.c_str());
        }
        h->has_prefixes = true;
    }
    if (!sfx.empty()) {
        if (!h->suffixes.build(std::move(sfx), 0, why)) {
            delete h;
            return fail(err, errlen, OG_E_FILTER, "%s", why.c_str());
        }
        h->has_suffixes = true;
    }
    *out = h;
    return OG_OK;
}

size_t og_filters_count(const og_filters* f) {
    return f ? (f->has_prefixes ? f->set.size() : 0) + (f->has_suffixes ? f->suffixes.size() : 0) : 0;
}

size_t og_filters_prefix_count(const og_filters* f) { return f && f->has_prefixes ? f->set.size() : 0; }

int og_filters_text(const og_filters* f, size_t i, char* out, size_t cap) {
    if (!f || i >= og_filters_count(f) || !out || cap == 0) return OG_E_ARG;
    const size_t np = og_filters_prefix_count(f);
    snprintf(out, cap, "%s", i < np ? f->set.filter(i).text.c_str() : f->suffixes.pattern(i - np).text.c_str());
    return OG_OK;
}

uint32_t og_filters_bits(const og_filters* f) { return f && f->has_prefixes ? f->set.bits() : 0; }

size_t og_filters_words(const og_filters* f, const uint64_t** words) {
    if (!f || !f->has_prefixes) return 0;
    if (words) *words = f->set.words().data();
    return f->set.words().size();
}

uint32_t og_filters_suffix_bits(const og_filters* f) { return f && f->has_suffixes ? f->suffixes.bits() : 0; }

size_t og_filters_suffix_words(const og_filters* f, const uint64_t** words) {
    if (!f || !f->has_suffixes) return 0;
    if (words) *words = f->suffixes.words().data();
    return f->suffixes.words().size();
}

long og_filters_match_address(const og_filters* f, const uint8_t pk[32]) {
    if (!f || !pk) return -1;
    if (f->has_prefixes) {
        const long m = f->set.match_key(pk);
        if (m >= 0) {
            const PrefixFilter& pf = f->set.filter((size_t)m);
            if (!pf.needs_full_check() || pf.matches_address(address(pk))) return m;
        }
    }
    if (f->has_suffixes) {
        uint8_t addr[35];
        address_bytes(pk, addr);
        const long j = f->suffixes.match_address(addr);
        if (j >= 0) return (long)og_filters_prefix_count(f) + j;
    }
    return -1;
}

double og_filters_occupancy(const og_filters* f) { return f ? f->set.occupancy() : 0.0; }

double og_filters_match_probability(const og_filters* f) {
    if (!f) return 0.0;
    std::vector<double> suffixes;
    for (size_t j = 0; f->has_suffixes && j < f->suffixes.size(); j++) suffixes.push_back(f->suffixes.pattern(j).probability());
    // the prefixes' and the suffixes' shares combine as the filters do
    return og::either_of({f->has_prefixes ? f->set.match_probability() : 0.0, og::either_of(suffixes)});
}

long og_filters_match(const og_filters* f, const uint8_t packed[32]) { return f ? f->set.match_key(packed) : -1; }

size_t og_filters_match_many(const og_filters* f, const uint8_t* packed, size_t n, size_t stride, int32_t* out) {
    if (!f || !packed || !out) return 0;
    size_t hits = 0;
    for (size_t i = 0; i < n; i++) {
        const long m = f->set.match_key(packed + i * stride);
        out[i] = (int32_t)m;
        if (m >= 0) hits++;
    }
    return hits;
}

void og_filters_free(og_filters* f) { delete f; }

}  // extern "C"
