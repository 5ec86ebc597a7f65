#include "filters.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "keys.h"

namespace og {

namespace {

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n')) a++;
    while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n')) b--;
    return s.substr(a, b - a);
}

uint64_t head64(const uint8_t packed[32]) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | packed[i];
    return v;
}

// top `bits` bits of the packed key, big-endian (src/filter.rs:2538-2549)
size_t slot_of(const uint8_t packed[32], uint32_t bits) { return (size_t)(head64(packed) >> (64 - bits)); }

}  // namespace

// Every slot of a `bits`-wide prefix index a pattern can occupy: the values its
// sets allow over the first bits / 5 symbols and the top bits % 5 bits of the
// next; false past 4096 slots (BitmapIndex::pattern_slots, src/filter.rs:2480-2530).
bool pattern_slots(const PrefixFilter& f, uint32_t bits, std::vector<uint32_t>& out) {
    const uint32_t full = bits / 5, rem = bits % 5;
    std::vector<uint32_t> values{0};
    for (uint32_t k = 0; k < full + (rem ? 1 : 0); k++) {
        const uint32_t set = k < f.sets.size() ? f.sets[k] : 0xffffffffu;
        uint32_t parts = 0;
        for (uint32_t v = 0; v < 32; v++)
            if ((set >> v) & 1) parts |= 1u << (k < full ? v : v >> (5 - rem));
        const size_t np = (size_t)__builtin_popcount(parts);
        if (values.size() * np > 4096) return false;
        const uint32_t shift = k < full ? bits - 5 * (k + 1) : 0;
        std::vector<uint32_t> next;
        next.reserve(values.size() * np);
        for (uint32_t base : values)
            for (uint32_t part = 0; part < 32; part++)
                if ((parts >> part) & 1) next.push_back(base | (part << shift));
        values.swap(next);
    }
    out.swap(values);
    return true;
}

bool PrefixFilter::matches_key(const uint8_t packed[32]) const {
    if (is_pattern()) {
        const size_t m = std::min(sets.size(), KEY_ONLY_SYMBOLS);
        for (size_t i = 0; i < m; i++)
            if (!((sets[i] >> symbol_at(packed, 32, i)) & 1)) return false;
        return true;
    }
    const size_t last = nbytes - 1;
    return std::memcmp(packed, bytes, last) == 0 && (packed[last] & mask) == bytes[last];
}

bool PrefixFilter::matches_address(const std::string& address) const {
    if (!is_pattern()) return address.compare(0, text.size(), text) == 0;
    if (address.size() < sets.size()) return false;
    for (size_t i = 0; i < sets.size(); i++) {
        const int v = base32_value(address[i]);
        if (v < 0 || !((sets[i] >> v) & 1)) return false;
    }
    return true;
}

bool parse_prefix(const std::string& raw, PrefixFilter& out, std::string& err) {
    std::string s = trim(raw);
    const size_t colon = s.find(':');
    if (colon != std::string::npos) {
        std::string form = trim(s.substr(0, colon));
        for (char& c : form) c = (char)std::tolower((unsigned char)c);
        if (form != "prefix") {
            err = "the " + form + " form is not supported by the device engine; only literal prefixes are";
            return false;
        }
        s = trim(s.substr(colon + 1));
    } else {
        size_t k = 0;
        while (k < s.size() && s[k] == '^') k++;
        s = s.substr(k);
    }
    if (s.empty()) {
        err = "the filter is empty";
        return false;
    }
    if (s.find_first_of("?[]") != std::string::npos) {
        // a pattern: wildcards or classes (Pattern::parse, src/filter.rs:298-350)
        std::vector<uint32_t> sets;
        if (!parse_symbol_sets(s, sets, err)) return false;
        if (sets.size() > ADDRESS_SYMBOLS) {
            err = "a filter of " + std::to_string(sets.size()) + " symbols is longer than an address (56)";
            return false;
        }
        if (std::all_of(sets.begin(), sets.end(), [](uint32_t x) { return x == 0xffffffffu; })) {
            err = "the filter fixes no symbol";
            return false;
        }
        out.sets = sets;
        out.text = render_sets(sets);
        out.nbytes = 0;
        out.mask = 0;
        std::memset(out.bytes, 0, sizeof out.bytes);
        return true;
    }
    out.sets.clear();
    if (s.size() > ADDRESS_SYMBOLS) {
        err = "a filter of " + std::to_string(s.size()) + " symbols is longer than an address (56)";
        return false;
    }
    std::string canon;
    for (size_t i = 0; i < s.size(); i++) {
        const int v = base32_value(s[i]);
        if (v < 0) {
            err = std::string("invalid character '") + s[i] + "' at position " + std::to_string(i) +
                  ": the base32 alphabet is a-z and 2-7";
            return false;
        }
        canon.push_back(BASE32_ALPHABET[v]);
    }
    out.text = canon;
    // decode the first min(len, 49) symbols into bytes plus a mask for the
    // partly significant last byte (src/filter.rs:649-685)
    const size_t sym = std::min(canon.size(), KEY_ONLY_SYMBOLS);
    const size_t bits = sym * 5;
    std::memset(out.bytes, 0, sizeof out.bytes);
    for (size_t i = 0; i < sym; i++) {
        const unsigned v = (unsigned)base32_value(canon[i]);
        for (unsigned k = 0; k < 5; k++) {
            const size_t b = i * 5 + k;
            if ((v >> (4 - k)) & 1) out.bytes[b / 8] |= (uint8_t)(0x80 >> (b % 8));
        }
    }
    out.nbytes = (bits + 7) / 8;
    const unsigned rem = bits % 8;
    out.mask = rem == 0 ? 0xff : (uint8_t)(0xff << (8 - rem));
    out.bytes[out.nbytes - 1] &= out.mask;
    return true;
}

bool parse_filter_lines(const char* text, std::vector<PrefixFilter>& prefixes, std::vector<SuffixPattern>& suffixes,
                        std::string& err) {
    const char* p = text;
    size_t line = 0;
    while (*p) {
        const char* e = std::strchr(p, '\n');
        const std::string s = e ? std::string(p, (size_t)(e - p)) : std::string(p);
        line++;
        const std::string t = trim(s);
        if (!t.empty()) {
            std::string why;
            const size_t colon = t.find(':');
            std::string form = colon == std::string::npos ? "" : trim(t.substr(0, colon));
            for (char& ch : form) ch = (char)std::tolower((unsigned char)ch);
            if (form == "suffix") {
                SuffixPattern sp;
                if (!parse_suffix(t.substr(colon + 1), sp, why)) {
                    err = "line " + std::to_string(line) + ": " + why;
                    return false;
                }
                suffixes.push_back(sp);
            } else {
                PrefixFilter f;
                if (!parse_prefix(t, f, why)) {
                    err = "line " + std::to_string(line) + ": " + why;
                    return false;
                }
                prefixes.push_back(f);
            }
        }
        if (!e) break;
        p = e + 1;
    }
    return true;
}

std::vector<uint64_t> build_bitmap(const std::vector<PrefixFilter>& filters, uint32_t bits) {
    std::vector<uint64_t> words;
    if (filters.empty() || bits < 8 || bits > 32) return words;
    words.assign((size_t)(((1ULL << bits) + 63) / 64), 0);
    for (const PrefixFilter& f : filters) {
        if (f.is_pattern()) {
            std::vector<uint32_t> slots;
            if (!pattern_slots(f, bits, slots)) return {};
            for (uint32_t v : slots) words[v >> 6] |= 1ULL << (v & 63);
            continue;
        }
        const size_t sym = std::min(f.text.size(), KEY_ONLY_SYMBOLS);
        const uint32_t pbits = (uint32_t)(sym * 5);
        uint8_t probe[32] = {0};
        std::memcpy(probe, f.bytes, f.nbytes);
        const size_t first = slot_of(probe, bits);
        const size_t run = pbits >= bits ? 1 : (size_t)1 << (bits - pbits);
        // whole words where the run covers them, bits at the ends
        size_t s = first;
        const size_t end = first + run;
        while (s < end && (s & 63)) {
            words[s >> 6] |= 1ULL << (s & 63);
            s++;
        }
        while (s + 64 <= end) {
            words[s >> 6] = ~0ULL;
            s += 64;
        }
        while (s < end) {
            words[s >> 6] |= 1ULL << (s & 63);
            s++;
        }
    }
    if (bitmap_occupancy(words, bits) > 0.25) words.clear();
    return words;
}

double bitmap_occupancy(const std::vector<uint64_t>& words, uint32_t bits) {
    uint64_t set = 0;
    for (uint64_t w : words) set += (uint64_t)__builtin_popcountll(w);
    return (double)set / (double)(1ULL << bits);
}

bool FilterSet::build(std::vector<PrefixFilter> filters, uint32_t bits, std::string& err) {
    std::sort(filters.begin(), filters.end(),
              [](const PrefixFilter& a, const PrefixFilter& b) { return a.text < b.text; });
    filters_.clear();
    long last_literal = -1;
    for (PrefixFilter& f : filters) {
        if (f.is_pattern()) {
            // patterns: exact duplicates only
            bool dup = false;
            for (const PrefixFilter& g : filters_) dup |= g.is_pattern() && g.text == f.text;
            if (!dup) filters_.push_back(f);
            continue;
        }
        // a literal prefix absorbs the literals it starts (src/filter.rs:1326-1339)
        if (last_literal >= 0) {
            const std::string& prev = filters_[(size_t)last_literal].text;
            if (f.text.compare(0, prev.size(), prev) == 0) continue;
        }
        last_literal = (long)filters_.size();
        filters_.push_back(f);
    }
    if (filters_.empty()) {
        err = "no filters";
        return false;
    }
    if (bits == 0) {
        std::vector<uint64_t> widest;
        uint32_t widest_bits = 0;
        for (uint32_t b = 16; b <= 24; b++) {
            std::vector<uint64_t> w = build_bitmap(filters_, b);
            if (w.empty()) continue;
            const bool good = bitmap_occupancy(w, b) <= 0.01;
            widest.swap(w);
            widest_bits = b;
            if (good) break;
        }
        words_.swap(widest);
        bits_ = widest_bits;
    } else {
        if (bits < 8 || bits > 32) {
            err = "the index width must be 8..32 bits";
            return false;
        }
        words_ = build_bitmap(filters_, bits);
        bits_ = bits;
    }
    if (words_.empty()) {
        err = "the filters fill more than a quarter of every index width; no bitmap can discriminate";
        return false;
    }
    // length buckets for the exact match
    buckets_.clear();
    patterns_.clear();
    for (size_t i = 0; i < filters_.size(); i++) {
        if (filters_[i].is_pattern()) {
            patterns_.push_back((uint32_t)i);
            continue;
        }
        const size_t sym = std::min(filters_[i].text.size(), KEY_ONLY_SYMBOLS);
        auto it = std::find_if(buckets_.begin(), buckets_.end(), [&](const Bucket& b) { return b.symbols == sym; });
        if (it == buckets_.end()) {
            Bucket b;
            b.symbols = sym;
            const unsigned hb = (unsigned)std::min<size_t>(sym * 5, 64);
            b.mask = hb == 64 ? ~0ULL : ~0ULL << (64 - hb);
            buckets_.push_back(b);
            it = buckets_.end() - 1;
        }
        uint8_t padded[32] = {0};
        std::memcpy(padded, filters_[i].bytes, filters_[i].nbytes);
        it->keys.push_back(head64(padded) & it->mask);
        it->owners.push_back((uint32_t)i);
    }
    for (Bucket& b : buckets_) {
        std::vector<size_t> order(b.keys.size());
        for (size_t k = 0; k < order.size(); k++) order[k] = k;
        std::sort(order.begin(), order.end(), [&](size_t x, size_t y) { return b.keys[x] < b.keys[y]; });
        std::vector<uint64_t> keys(order.size());
        std::vector<uint32_t> owners(order.size());
        for (size_t k = 0; k < order.size(); k++) {
            keys[k] = b.keys[order[k]];
            owners[k] = b.owners[order[k]];
        }
        b.keys.swap(keys);
        b.owners.swap(owners);
    }
    return true;
}

double FilterSet::occupancy() const { return words_.empty() ? 0.0 : bitmap_occupancy(words_, bits_); }

bool FilterSet::may_match(const uint8_t packed[32]) const {
    if (words_.empty()) return false;  // a set with no prefixes
    const size_t s = slot_of(packed, bits_);
    return (words_[s >> 6] >> (s & 63)) & 1;
}

long FilterSet::match_key(const uint8_t packed[32]) const {
    if (!may_match(packed)) return -1;
    const uint64_t head = head64(packed);
    for (const Bucket& b : buckets_) {
        const uint64_t probe = head & b.mask;
        auto lo = std::lower_bound(b.keys.begin(), b.keys.end(), probe);
        for (auto it = lo; it != b.keys.end() && *it == probe; ++it) {
            const uint32_t owner = b.owners[(size_t)(it - b.keys.begin())];
            if (filters_[owner].matches_key(packed)) return (long)owner;
        }
    }
    for (uint32_t i : patterns_)
        if (filters_[i].matches_key(packed)) return (long)i;
    return -1;
}

void FilterSet::device_tables(std::vector<DeviceBucket>& buckets, std::vector<uint64_t>& keys,
                              std::vector<uint32_t>& owners) const {
    buckets.clear();
    keys.clear();
    owners.clear();
    std::vector<std::vector<std::pair<uint64_t, uint32_t>>> by_len(DEVICE_SYMBOLS + 1);
    for (size_t i = 0; i < filters_.size(); i++) {
        if (filters_[i].is_pattern()) continue;
        const size_t sym = std::min(filters_[i].text.size(), DEVICE_SYMBOLS);
        const uint32_t hb = (uint32_t)(sym * 5);
        uint8_t padded[32] = {0};
        std::memcpy(padded, filters_[i].bytes, filters_[i].nbytes);
        by_len[sym].push_back({head64(padded) & (~0ULL << (64 - hb)), (uint32_t)i});
    }
    for (size_t sym = 1; sym <= DEVICE_SYMBOLS; sym++) {
        auto& v = by_len[sym];
        if (v.empty()) continue;
        std::sort(v.begin(), v.end());
        buckets.push_back(DeviceBucket{(uint32_t)(sym * 5), (uint32_t)keys.size(), (uint32_t)v.size()});
        for (auto& kv : v) {
            keys.push_back(kv.first);
            owners.push_back(kv.second);
        }
    }
}

void FilterSet::device_patterns(std::vector<uint32_t>& rows) const {
    rows.clear();
    for (uint32_t i : patterns_) {
        const PrefixFilter& f = filters_[i];
        std::vector<uint32_t> row(PATTERN_ROW, 0xffffffffu);
        row[0] = i;
        row[1] = (uint32_t)std::min(f.sets.size(), KEY_ONLY_SYMBOLS);
        for (size_t k = 0; k < row[1]; k++) row[2 + k] = f.sets[k];
        rows.insert(rows.end(), row.begin(), row.end());
    }
}

double FilterSet::match_probability() const {
    // each kept filter anchored at the start, every symbol it names, the
    // tail's protocol rooms included; combined as the reference does
    std::vector<double> p;
    p.reserve(filters_.size());
    for (const PrefixFilter& f : filters_) {
        if (f.is_pattern()) {
            p.push_back(anchored_probability(f.sets.data(), f.sets.size(), 0));
        } else {
            std::vector<uint32_t> sets(f.text.size());
            for (size_t i = 0; i < f.text.size(); i++) sets[i] = 1u << base32_value(f.text[i]);
            p.push_back(anchored_probability(sets.data(), sets.size(), 0));
        }
    }
    return either_of(p);
}

}  // namespace og
