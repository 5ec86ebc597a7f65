// Suffix filters and the suffix bitmap the device tests.
//
// Follows src/filter.rs for the `suffix:` form: a symbol set per position
// (literal symbols, `?` and `[...]` classes with ranges, parse_symbols
// :495-560), the reachability check of the address tail (the last symbol
// is always `d`, the one before it one of `aiqy`: check_reachable_tail
// :566-600), and the suffix bitmap (BitmapIndex::build_over_suffixes and
// suffix_slots, :2393-2480): the index is keyed on the last `bits` bits of
// the key-derived span (base32 bits [255 - bits, 255) of the packed key), a
// suffix fills every slot its symbols allow there, and symbol 49, which the
// deferred sign bit touches, is widened to both sign values (either_sign,
// :144-164). The width is the narrowest of 16..24 whose occupancy stays
// under 1% divided by the number of suffixes, else the widest that is at
// most a quarter full (narrowest_acceptable / target_for_walk,
// :2257-2300).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace og {

constexpr size_t KEY_DERIVED_SYMBOLS = 51;  // symbols 0..50 come from the key alone
constexpr size_t SIGN_SYMBOL = 49;          // the symbol the sign bit (base32 bit 248) lands in

// Symbol `position` (five bits, most significant first) of a big-endian bit
// string of `len` bytes; bits past the end read as zero.
uint32_t symbol_at(const uint8_t* bytes, size_t len, size_t position);

// The share of addresses whose symbols from `start` on fall in `sets`: per
// position, the accepted symbols the protocol can produce there over the
// symbols it can produce there (the last symbol is always 'd', the one
// before it one of 'a', 'i', 'q', 'y'), multiplied over the positions
// (Pattern::probability_at with protocol_allows, src/filter.rs:443-452,
// 226-238).
double anchored_probability(const uint32_t* sets, size_t n, size_t start);

struct SuffixPattern {
    std::string text;             // canonical: "suffix:" + the body, lowercase
    std::vector<uint32_t> sets;   // bit v set = symbol value v allowed; position 56 - size() + i
    size_t start() const { return 56 - sets.size(); }
    // The exact check on the 35 bytes pk || checksum || version.
    bool matches_address(const uint8_t addr[35]) const;
    // The share of addresses this suffix matches.
    double probability() const { return anchored_probability(sets.data(), sets.size(), start()); }
    // The part a packed key (sign bit unknown) can decide: every position
    // below 51 the suffix reaches, with symbol 49 widened to both signs.
    bool key_prefilter(const uint8_t packed[32]) const;
};

// A filter body as one symbol set per position: literal symbols, `?` (any)
// and `[...]` classes with `a-e` ranges (parse_symbols, src/filter.rs:495-560).
bool parse_symbol_sets(const std::string& body, std::vector<uint32_t>& sets, std::string& err);
// The canonical text of symbol sets: a symbol, `?`, or the class's members.
std::string render_sets(const std::vector<uint32_t>& sets);

// Parses the body of a `suffix:` filter (without the form name).
bool parse_suffix(const std::string& body, SuffixPattern& out, std::string& err);

class SuffixSet {
public:
    // bits == 0 chooses the width. Fails when no width covers every suffix
    // within a quarter of the slots: a suffix too short to reach into the key
    // would fill the whole index, and the device would keep every candidate.
    bool build(std::vector<SuffixPattern> patterns, uint32_t bits, std::string& err);

    size_t size() const { return patterns_.size(); }
    const SuffixPattern& pattern(size_t i) const { return patterns_[i]; }
    uint32_t bits() const { return bits_; }
    uint32_t offset() const { return 255 - bits_; }  // first base32 bit of the window
    const std::vector<uint64_t>& words() const { return words_; }
    double occupancy() const;
    bool may_match(const uint8_t packed[32]) const;
    // Index of the first suffix the full address matches, or -1.
    long match_address(const uint8_t addr[35]) const;

    // Every slot a suffix occupies in a window of `bits` at the end of the
    // key-derived span; false when there are more than 4096 of them.
    static bool slots(const SuffixPattern& p, uint32_t bits, std::vector<uint32_t>& out);

private:
    std::vector<SuffixPattern> patterns_;
    std::vector<uint64_t> words_;
    uint32_t bits_ = 0;
};

// 1 - prod(1 - p) over a set's filters, kept small where p is (FilterSet::
// probability, src/filter.rs:1979-1990, with log1p / expm1).
double either_of(const std::vector<double>& p);

// The 35 address bytes of a full public key: pk || checksum || 0x03.
void address_bytes(const uint8_t pk[32], uint8_t out[35]);

}  // namespace og
