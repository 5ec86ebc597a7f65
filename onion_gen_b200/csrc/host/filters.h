// Address-prefix filters and the prefix bitmap the device tests.
//
// Follows src/filter.rs for the prefix form: Filter::parse (bytes + mask of the
// first min(len, 49) symbols, :649-685), FilterSet::new (sort, drop duplicates
// and absorbed filters, :1326-1339), BitmapIndex (slot = top `bits` bits of the
// packed key read big-endian, a prefix shorter than the index fills a run,
// :2321-2604), the width choice (narrowest 16..24 at <= 1% occupancy, else the
// widest that is <= 25% full, :2279-2295) and the exact match behind the bitmap
// (length buckets with a binary search, :2645-2700). Prefixes with `?` and
// `[...]` classes fill the slots their symbol sets allow (pattern_slots,
// :2480-2530) and are matched after the literals, in order. Suffixes live in
// suffix.h; substrings and regular expressions are not part of this engine.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "suffix.h"

namespace og {

constexpr size_t KEY_ONLY_SYMBOLS = 49;
constexpr size_t ADDRESS_SYMBOLS = 56;

struct PrefixFilter {
    std::string text;  // canonical: lowercase symbols; a pattern's `?` and classes rendered
    uint8_t bytes[32];  // a literal's first min(len, 49) symbols decoded
    size_t nbytes;
    uint8_t mask;
    std::vector<uint32_t> sets;  // a pattern's symbol set per position; empty for a literal
    bool is_pattern() const { return !sets.empty(); }
    size_t symbols() const { return is_pattern() ? sets.size() : text.size(); }
    // filters longer than the key-only span need the full address checked
    bool needs_full_check() const { return symbols() > KEY_ONLY_SYMBOLS; }
    // the key-only part: a masked byte compare, or a pattern's sets over the
    // first min(len, 49) symbols
    bool matches_key(const uint8_t packed[32]) const;
    // the full check on an address text of 56 symbols
    bool matches_address(const std::string& address) const;
};

// Parses one filter; returns false and an explanation on error.
bool parse_prefix(const std::string& raw, PrefixFilter& out, std::string& err);

class FilterSet {
public:
    // bits == 0 chooses the width; otherwise 8..32.
    bool build(std::vector<PrefixFilter> filters, uint32_t bits, std::string& err);

    size_t size() const { return filters_.size(); }
    const PrefixFilter& filter(size_t i) const { return filters_[i]; }
    uint32_t bits() const { return bits_; }
    const std::vector<uint64_t>& words() const { return words_; }
    double occupancy() const;
    bool may_match(const uint8_t packed[32]) const;
    // index of the matching filter or -1; at most one matches because no kept
    // filter is a prefix of another.
    long match_key(const uint8_t packed[32]) const;
    // expected fraction of candidates that match some filter exactly
    double match_probability() const;

    // The exact-match tables in the form the device searches: one bucket
    // per distinct length (capped at DEVICE_SYMBOLS symbols), each a sorted
    // run of masked 64-bit key heads with the owning filter's index.
    // Filters longer than DEVICE_SYMBOLS are matched on their first
    // DEVICE_SYMBOLS symbols there and confirmed by match_key() on the host.
    static constexpr size_t DEVICE_SYMBOLS = 12;
    struct DeviceBucket {
        uint32_t bits;    // significant leading bits of the head
        uint32_t offset;  // into keys / owners
        uint32_t count;
    };
    void device_tables(std::vector<DeviceBucket>& buckets, std::vector<uint64_t>& keys,
                       std::vector<uint32_t>& owners) const;
    // The patterns in the form the device walks after the buckets, in index
    // order: per pattern PATTERN_ROW words, its filter index, the number of
    // key-only symbols it fixes (at most 49) and one set per position.
    static constexpr size_t PATTERN_ROW = 2 + KEY_ONLY_SYMBOLS;
    void device_patterns(std::vector<uint32_t>& rows) const;

private:
    struct Bucket {
        size_t symbols;
        uint64_t mask;
        std::vector<uint64_t> keys;
        std::vector<uint32_t> owners;
    };
    std::vector<PrefixFilter> filters_;
    std::vector<uint64_t> words_;
    uint32_t bits_ = 0;
    std::vector<Bucket> buckets_;
    std::vector<uint32_t> patterns_;  // indices of the patterns, in order
};

bool pattern_slots(const PrefixFilter& f, uint32_t bits, std::vector<uint32_t>& out);

// Parses newline-separated filters: `suffix:` lines into `suffixes`, the
// rest (bare, `^` or `prefix:`) into `prefixes`. Blank lines are skipped;
// an error names its line.
bool parse_filter_lines(const char* text, std::vector<PrefixFilter>& prefixes, std::vector<SuffixPattern>& suffixes,
                        std::string& err);

// Builds the bitmap over `filters` at `bits`; empty when more than a quarter
// of the slots would be set.
std::vector<uint64_t> build_bitmap(const std::vector<PrefixFilter>& filters, uint32_t bits);
double bitmap_occupancy(const std::vector<uint64_t>& words, uint32_t bits);

}  // namespace og

// The C ABI's filter-set handle (og_filters_new), shared with the engine's
// device exact match: the literal prefixes and the suffixes of one set.
// Filter index i < set.size() is prefix i; set.size() + j is suffix j.
struct og_filters {
    og::FilterSet set;
    og::SuffixSet suffixes;
    bool has_prefixes = false;
    bool has_suffixes = false;
};
