// The launch-shape cache, tuning.yaml (src/tuning.rs).
//
// Same file, format and key as the reference: `format: 1`, a map `entries`
// from `device/<name with '/' and '\n' replaced by '_'>/<api>/<threads>/<version>`
// (src/tuning.rs:65-74) to a Shape {first, second, rate, at}
// (src/tuning.rs:27-39), stored under $XDG_CACHE_HOME/onion-gen/ or
// ~/.cache/onion-gen/ (src/tuning.rs:80-91) and written beside then renamed
// (src/tuning.rs:103-125). For this engine `first` is the inversion batch
// (`half`, a round being 2*half+1 candidates), `second` the lanes in flight;
// `block`, `rounds` and `lanes_per_thread` ride along as extra fields, which
// the reference's reader ignores. Every failure is "no entry", never an error.
#pragma once
#include <cstdint>
#include <string>

namespace og {

struct Shape {
    uint32_t first = 0;
    uint32_t second = 0;
    double rate = 0;
    int64_t at = 0;
    uint32_t block = 0;
    uint32_t rounds = 0;
    uint32_t lanes_per_thread = 0;
};

extern const char* const ENGINE_VERSION;

std::string tuning_path();
std::string device_key(const std::string& name, const std::string& api, uint32_t threads);
bool tuning_get(const std::string& key, Shape& out);
void tuning_put(const std::string& key, const Shape& shape);
int64_t unix_now();

}  // namespace og
