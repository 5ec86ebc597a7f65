// og_serve: continuous batching of search requests over one og_batch.
//
// One worker thread owns the batch. Submissions go to a FIFO queue under a
// mutex; the worker admits from its head while the batch has room (it stops
// at the first request the memory budget cannot take, so admission stays in
// arrival order), runs a step, and completes every request whose quota is
// met: its hits are copied out, its completion is stamped when that step's
// results are taken, and it is retired so its lanes and tables go to the
// next requests. The batch keeps a second step in flight meanwhile, so the
// worker's admissions and completions overlap the device's work.
#include <time.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/onion_gen_b200.h"
#include "common.h"

namespace {

uint64_t now_ns() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (uint64_t)ts.tv_sec * 1000000000ULL + (uint64_t)ts.tv_nsec;
}

struct Request {
    uint64_t id;
    uint8_t seed[32];
    std::string filters;
    uint32_t quota;
    uint64_t arrival_ns;
    uint64_t admit_ns = 0;
};

}  // namespace

struct og_serve {
    og_batch* batch = nullptr;
    uint32_t max_running = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    std::deque<Request> queue;                          // guarded by mu
    std::vector<og_serve_done> done;                    // guarded by mu
    std::map<uint64_t, std::vector<og_batch_hit>> results;  // guarded by mu
    og_serve_stats stats{};                             // guarded by mu
    // worker-only state
    std::map<uint64_t, Request> running;

    void complete(const Request& r, uint32_t status, uint64_t candidates, std::vector<og_batch_hit>&& hits) {
        og_serve_done d{};
        d.request_id = r.id;
        d.arrival_ns = r.arrival_ns;
        d.admit_ns = r.admit_ns;
        d.done_ns = now_ns();
        d.candidates = candidates;
        d.hits = (uint32_t)hits.size();
        d.status = status;
        std::lock_guard<std::mutex> lock(mu);
        done.push_back(d);
        results[r.id] = std::move(hits);
        stats.completed++;
    }

    void admit() {
        for (;;) {
            Request r;
            {
                std::lock_guard<std::mutex> lock(mu);
                if (queue.empty() || running.size() >= max_running) return;
                r = queue.front();
            }
            char err[256];
            const int rc = og_batch_admit(batch, r.id, r.seed, r.filters.c_str(), r.quota, err, sizeof err);
            if (rc == OG_E_NOMEM || rc == OG_E_CAPACITY) {
                if (!running.empty()) return;  // wait for room, in arrival order
                // nothing running and still no room: it can never be admitted
            }
            {
                std::lock_guard<std::mutex> lock(mu);
                queue.pop_front();
            }
            if (rc != OG_OK) {
                complete(r, (uint32_t)rc, 0, {});
                continue;
            }
            r.admit_ns = now_ns();
            running[r.id] = r;
            std::lock_guard<std::mutex> lock(mu);
            stats.running = running.size();
        }
    }

    void loop() {
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(mu);
                cv.wait(lock, [&] { return stop || !queue.empty() || !running.empty(); });
                if (stop) return;
            }
            admit();
            if (running.empty()) continue;
            size_t n = 0;
            char err[256];
            // the step's hits stay in the batch; a request's come out of
            // og_batch_results when it completes
            const int rc = og_batch_step(batch, nullptr, 0, &n, err, sizeof err);
            const double ms = og_batch_last_step_ms(batch);
            const uint64_t cand = og_batch_last_step_candidates(batch);
            {
                std::lock_guard<std::mutex> lock(mu);
                stats.steps++;
                stats.candidates += cand;
                stats.device_ms += ms;
            }
            // collect finished requests. A hit that did not re-derive
            // (OG_E_VERIFY) ends only its own search, which completes with
            // that status; any other failure closes the batch, and every
            // running request ends with it.
            const bool batch_failed = rc != OG_OK && rc != OG_E_VERIFY;
            std::vector<uint64_t> finished;
            for (auto& kv : running) {
                og_search_status st;
                if (og_batch_status(batch, kv.first, &st) != OG_OK) continue;
                if (batch_failed || st.done) {
                    std::vector<og_batch_hit> hits(st.quota);
                    size_t got = 0;
                    og_batch_results(batch, kv.first, hits.data(), hits.size(), &got);
                    hits.resize(got);
                    complete(kv.second, batch_failed ? (uint32_t)rc : st.status, st.candidates, std::move(hits));
                    finished.push_back(kv.first);
                }
            }
            for (uint64_t id : finished) {
                og_batch_retire(batch, id);
                running.erase(id);
            }
            std::lock_guard<std::mutex> lock(mu);
            stats.running = running.size();
        }
    }
};

extern "C" {

uint64_t og_serve_now_ns(void) { return now_ns(); }

int og_serve_new(int ordinal, const og_serve_config* cfg, og_serve** out, char* err, size_t errlen) {
    if (!out) return og::fail(err, errlen, OG_E_ARG, "null argument");
    *out = nullptr;
    og_serve_config c{};
    if (cfg) c = *cfg;
    og_serve* s = new (std::nothrow) og_serve();
    if (!s) return og::fail(err, errlen, OG_E_NOMEM, "host memory");
    const int rc = og_batch_new(ordinal, &c.batch, &s->batch, err, errlen);
    if (rc != OG_OK) {
        delete s;
        return rc;
    }
    s->max_running = c.max_running ? c.max_running : (c.batch.max_searches ? c.batch.max_searches : 4096);
    s->worker = std::thread([s] { s->loop(); });
    *out = s;
    return OG_OK;
}

int og_serve_submit(og_serve* s, uint64_t request_id, const uint8_t seed[32], const char* filters, uint32_t quota,
                    char* err, size_t errlen) {
    if (!s || !seed || !filters) return og::fail(err, errlen, OG_E_ARG, "null argument");
    if (quota == 0) return og::fail(err, errlen, OG_E_ARG, "a quota of zero");
    Request r;
    r.id = request_id;
    std::memcpy(r.seed, seed, 32);
    r.filters = filters;
    r.quota = quota;
    r.arrival_ns = now_ns();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->queue.push_back(std::move(r));
    }
    s->cv.notify_one();
    return OG_OK;
}

int og_serve_poll(og_serve* s, og_serve_done* out, size_t cap, size_t* n) {
    if (!s || !n) return OG_E_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    const size_t m = std::min(cap, s->done.size());
    for (size_t i = 0; i < m; i++) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + (long)m);
    *n = m;
    return OG_OK;
}

int og_serve_results(og_serve* s, uint64_t request_id, og_batch_hit* out, size_t cap, size_t* n) {
    if (!s || !n) return OG_E_ARG;
    *n = 0;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->results.find(request_id);
    if (it == s->results.end()) return OG_E_STATE;
    if (cap < it->second.size()) return OG_E_CAPACITY;
    for (size_t i = 0; i < it->second.size(); i++) out[i] = it->second[i];
    *n = it->second.size();
    s->results.erase(it);
    return OG_OK;
}

void og_serve_stats_get(og_serve* s, og_serve_stats* st) {
    if (!s || !st) return;
    std::lock_guard<std::mutex> lock(s->mu);
    *st = s->stats;
    st->queued = s->queue.size();
}

void og_serve_free(og_serve* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    og_batch_free(s->batch);
    delete s;
}

}  // extern "C"
