#include "suffix.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "keys.h"

namespace og {

namespace {

constexpr uint32_t ALL = 0xffffffffu;
constexpr size_t ADDRESS_LEN = 56;
constexpr size_t SLOT_BUDGET = 4096;  // past this many slots one suffix fills the map alone

// The same set plus every value that differs from a member only in the sign
// bit, which is worth 2 within symbol 49 (bits 245..249, the sign at 248).
uint32_t either_sign(uint32_t set) { return set | ((set & 0x33333333u) << 2) | ((set & 0xccccccccu) >> 2); }

std::string render(const std::vector<uint32_t>& sets) { return "suffix:" + render_sets(sets); }

std::string where(size_t i) { return " at position " + std::to_string(i); }

}  // namespace

uint32_t symbol_at(const uint8_t* bytes, size_t len, size_t position) {
    const size_t bit = position * 5, byte = bit / 8, shift = bit % 8;
    const uint32_t hi = byte < len ? (uint32_t)bytes[byte] << 8 : 0;
    const uint32_t lo = byte + 1 < len ? bytes[byte + 1] : 0;
    return ((hi | lo) >> (11 - shift)) & 0x1f;
}

bool SuffixPattern::matches_address(const uint8_t addr[35]) const {
    const size_t s = start();
    for (size_t i = 0; i < sets.size(); i++)
        if (!((sets[i] >> symbol_at(addr, 35, s + i)) & 1)) return false;
    return true;
}

bool SuffixPattern::key_prefilter(const uint8_t packed[32]) const {
    const size_t s = start();
    for (size_t i = 0; i < sets.size() && s + i < KEY_DERIVED_SYMBOLS; i++) {
        const size_t at = s + i;
        const uint32_t set = at == SIGN_SYMBOL ? either_sign(sets[i]) : sets[i];
        if (!((set >> symbol_at(packed, 32, at)) & 1)) return false;
    }
    return true;
}

bool parse_symbol_sets(const std::string& body, std::vector<uint32_t>& sets, std::string& err) {
    sets.clear();
    for (size_t i = 0; i < body.size();) {
        const char c = body[i];
        if (c == '?') {
            sets.push_back(ALL);
            i++;
        } else if (c == '[') {
            const size_t end = body.find(']', i);
            if (end == std::string::npos) {
                err = "an unbalanced '['" + where(i);
                return false;
            }
            uint32_t set = 0;
            for (size_t j = i + 1; j < end;) {
                const int first = base32_value(body[j]);
                if (first < 0) {
                    err = std::string("invalid character '") + body[j] + "'" + where(j);
                    return false;
                }
                if (j + 2 < end && body[j + 1] == '-') {
                    const int last = base32_value(body[j + 2]);
                    if (last < 0) {
                        err = std::string("invalid character '") + body[j + 2] + "'" + where(j + 2);
                        return false;
                    }
                    if (last < first) {
                        err = "an empty range" + where(j);
                        return false;
                    }
                    for (int v = first; v <= last; v++) set |= 1u << v;
                    j += 3;
                } else {
                    set |= 1u << first;
                    j++;
                }
            }
            if (set == 0) {
                err = "an empty class" + where(i);
                return false;
            }
            sets.push_back(set);
            i = end + 1;
        } else if (c == ']') {
            err = "an unbalanced ']'" + where(i);
            return false;
        } else {
            const int v = base32_value(c);
            if (v < 0) {
                err = std::string("invalid character '") + c + "'" + where(i) + ": the base32 alphabet is a-z and 2-7";
                return false;
            }
            sets.push_back(1u << v);
            i++;
        }
    }
    return true;
}

std::string render_sets(const std::vector<uint32_t>& sets) {
    std::string s;
    for (uint32_t set : sets) {
        if (set == ALL) {
            s.push_back('?');
        } else if (__builtin_popcount(set) == 1) {
            s.push_back(BASE32_ALPHABET[__builtin_ctz(set)]);
        } else {
            s.push_back('[');
            for (int v = 0; v < 32; v++)
                if ((set >> v) & 1) s.push_back(BASE32_ALPHABET[v]);
            s.push_back(']');
        }
    }
    return s;
}

bool parse_suffix(const std::string& raw, SuffixPattern& out, std::string& err) {
    size_t a = 0, b = raw.size();
    while (a < b && (raw[a] == ' ' || raw[a] == '\t' || raw[a] == '\r')) a++;
    while (b > a && (raw[b - 1] == ' ' || raw[b - 1] == '\t' || raw[b - 1] == '\r')) b--;
    const std::string body = raw.substr(a, b - a);
    std::vector<uint32_t> sets;
    if (!parse_symbol_sets(body, sets, err)) return false;
    if (sets.empty()) {
        err = "the filter is empty";
        return false;
    }
    if (sets.size() > ADDRESS_LEN) {
        err = "a suffix of " + std::to_string(sets.size()) + " symbols is longer than an address (56)";
        return false;
    }
    if (std::all_of(sets.begin(), sets.end(), [](uint32_t s) { return s == ALL; })) {
        err = "the suffix fixes no symbol";
        return false;
    }
    // the tail of a v3 address: the version byte makes the last symbol 'd'
    // and leaves the one before it one of 'a', 'i', 'q', 'y'
    if (!((sets.back() >> base32_value('d')) & 1)) {
        err = "no v3 address ends in '" + render({sets.back()}).substr(7) + "': the last symbol is always 'd'";
        return false;
    }
    if (sets.size() >= 2) {
        const uint32_t tail = (1u << base32_value('a')) | (1u << base32_value('i')) | (1u << base32_value('q')) |
                              (1u << base32_value('y'));
        if (!(sets[sets.size() - 2] & tail)) {
            err = "the second-to-last symbol of a v3 address is one of 'a', 'i', 'q', 'y'";
            return false;
        }
    }
    out.sets = sets;
    out.text = render(sets);
    return true;
}

double anchored_probability(const uint32_t* sets, size_t n, size_t start) {
    const uint32_t last = 1u << base32_value('d');
    const uint32_t penultimate = (1u << base32_value('a')) | (1u << base32_value('i')) | (1u << base32_value('q')) |
                                 (1u << base32_value('y'));
    double p = 1.0;
    for (size_t i = 0; i < n; i++) {
        const size_t pos = start + i;
        const uint32_t room = pos + 1 == ADDRESS_LEN ? last : pos + 2 == ADDRESS_LEN ? penultimate : ALL;
        p *= (double)__builtin_popcount(sets[i] & room) / (double)__builtin_popcount(room);
    }
    return p;
}

double either_of(const std::vector<double>& p) {
    double log_miss = 0.0;
    for (double q : p) log_miss += std::log1p(-q);
    return -std::expm1(log_miss);
}

bool SuffixSet::slots(const SuffixPattern& p, uint32_t bits, std::vector<uint32_t>& out) {
    const size_t window_lo = 255 - bits, window_hi = 255;
    const size_t start = p.start();
    std::vector<uint32_t> values{0};
    for (size_t symbol = window_lo / 5; symbol <= (window_hi - 1) / 5; symbol++) {
        const size_t lo = std::max(symbol * 5, window_lo), hi = std::min(symbol * 5 + 5, window_hi);
        const size_t width = hi - lo, shift = window_hi - hi;
        uint32_t set = symbol >= start ? p.sets[symbol - start] : ALL;
        if (symbol == SIGN_SYMBOL) set = either_sign(set);
        // the distinct values of the part of this symbol inside the window
        uint32_t seen = 0;
        std::vector<uint32_t> parts;
        for (uint32_t v = 0; v < 32; v++) {
            if (!((set >> v) & 1)) continue;
            const uint32_t part = (v >> (5 - (hi - symbol * 5))) & ((1u << width) - 1);
            if (!((seen >> part) & 1)) {
                seen |= 1u << part;
                parts.push_back(part);
            }
        }
        std::sort(parts.begin(), parts.end());
        if (values.size() * parts.size() > SLOT_BUDGET) return false;
        std::vector<uint32_t> next;
        next.reserve(values.size() * parts.size());
        for (uint32_t base : values)
            for (uint32_t part : parts) next.push_back(base | (part << shift));
        values.swap(next);
    }
    out.swap(values);
    return true;
}

namespace {

// The bitmap over every suffix at one width; empty when a suffix has too many
// slots or the map is more than a quarter full.
std::vector<uint64_t> suffix_bitmap(const std::vector<SuffixPattern>& patterns, uint32_t bits) {
    std::vector<uint64_t> words((size_t)(((1ULL << bits) + 63) / 64), 0);
    std::vector<uint32_t> s;
    for (const SuffixPattern& p : patterns) {
        if (!SuffixSet::slots(p, bits, s)) return {};
        for (uint32_t v : s) words[v >> 6] |= 1ULL << (v & 63);
    }
    uint64_t set = 0;
    for (uint64_t w : words) set += (uint64_t)__builtin_popcountll(w);
    if ((double)set / (double)(1ULL << bits) > 0.25) return {};
    return words;
}

double occupancy_of(const std::vector<uint64_t>& words, uint32_t bits) {
    uint64_t set = 0;
    for (uint64_t w : words) set += (uint64_t)__builtin_popcountll(w);
    return (double)set / (double)(1ULL << bits);
}

}  // namespace

bool SuffixSet::build(std::vector<SuffixPattern> patterns, uint32_t bits, std::string& err) {
    std::sort(patterns.begin(), patterns.end(),
              [](const SuffixPattern& a, const SuffixPattern& b) { return a.text < b.text; });
    patterns_.clear();
    for (SuffixPattern& p : patterns)
        if (patterns_.empty() || patterns_.back().text != p.text) patterns_.push_back(p);
    if (patterns_.empty()) {
        err = "no suffixes";
        return false;
    }
    words_.clear();
    bits_ = 0;
    if (bits == 0) {
        const double target = 0.01 / (double)patterns_.size();
        for (uint32_t b = 16; b <= 24; b++) {
            std::vector<uint64_t> w = suffix_bitmap(patterns_, b);
            if (w.empty()) continue;
            const bool good = occupancy_of(w, b) <= target;
            words_.swap(w);
            bits_ = b;
            if (good) break;
        }
    } else {
        if (bits < 8 || bits > 32) {
            err = "the index width must be 8..32 bits";
            return false;
        }
        words_ = suffix_bitmap(patterns_, bits);
        bits_ = words_.empty() ? 0 : bits;
    }
    if (words_.empty()) {
        err = "a suffix reaches too little of the key for a suffix bitmap (the device needs one that fixes "
              "about 13 bits of symbols 46..50, i.e. 8 symbols or more)";
        return false;
    }
    return true;
}

double SuffixSet::occupancy() const { return words_.empty() ? 0.0 : occupancy_of(words_, bits_); }

bool SuffixSet::may_match(const uint8_t packed[32]) const {
    if (words_.empty()) return false;
    const uint32_t off = offset(), byte = off / 8, within = off % 8;
    uint64_t word = 0;
    for (uint32_t i = 0; i < 8; i++) word = (word << 8) | (byte + i < 32 ? packed[byte + i] : 0);
    const uint64_t slot = (word << within) >> (64 - bits_);
    return (words_[slot >> 6] >> (slot & 63)) & 1;
}

long SuffixSet::match_address(const uint8_t addr[35]) const {
    for (size_t i = 0; i < patterns_.size(); i++)
        if (patterns_[i].matches_address(addr)) return (long)i;
    return -1;
}

void address_bytes(const uint8_t pk[32], uint8_t out[35]) {
    std::memcpy(out, pk, 32);
    checksum(pk, out + 32);
    out[34] = 0x03;
}

}  // namespace og
