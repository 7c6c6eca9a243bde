// Serving load generator (benchmark harness, not part of the library).
//
// Drives sort requests of a pool of device-resident arrays into either the
// b200sort server (continuous batching) or per-request plain launches
// (b200s_sort_packed with arrays = 1, one launch per request on one stream),
// in two ways:
//   * open loop: Poisson arrivals at a given rate for a given time; latency
//     runs from each request's scheduled arrival to its result being written;
//   * closed loop: a fixed number of requests kept outstanding, as fast as
//     the system completes them: its throughput is the peak sustained rate.
// Request i uses pool entry i % pool.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <random>
#include <thread>
#include <vector>

#include "b200sort.h"

namespace {

inline int64_t now_ns() { return b200s_server_clock_ns(); }

struct Percentiles {
    double p50 = 0, p99 = 0, p999 = 0, max = 0, mean = 0;
};

Percentiles percentiles(std::vector<int64_t>& v) {
    Percentiles p;
    if (v.empty()) return p;
    auto at = [&](double q) {
        const size_t k = size_t(q * double(v.size() - 1) + 0.5);
        std::nth_element(v.begin(), v.begin() + long(k), v.end());
        return double(v[k]) * 1e-3;
    };
    p.p50 = at(0.5);
    p.p99 = at(0.99);
    p.p999 = at(0.999);
    p.max = double(*std::max_element(v.begin(), v.end())) * 1e-3;
    double s = 0;
    for (int64_t x : v) s += double(x);
    p.mean = s / double(v.size()) * 1e-3;
    return p;
}

}  // namespace

extern "C" {

typedef struct lg_result {
    int64_t submitted, completed, rejected, batches, peak_arena_bytes;
    double p50_us, p99_us, p999_us, max_us, mean_us;
    double span_s;            // first arrival -> last completion
    double keys_per_s;        // keys completed / span
    double req_per_s;         // requests completed / span
    double offered_req_per_s; // arrival rate asked for (open loop)
    double max_lag_us;        // latest a submission ran behind its scheduled arrival
    double mean_batch;
    int32_t overloaded;       // submissions fell behind by more than max_lag_s: stopped early
} lg_result;

enum { LG_SERVER_OPEN = 0, LG_PLAIN_OPEN = 1, LG_SERVER_CLOSED = 2, LG_PLAIN_CLOSED = 3 };

// mode: LG_*.  rate/duration_s: open loop.  window: outstanding requests
// (closed loop).  Returns 0, or the failing b200s_status / CUDA error + 1000.
int lg_run(int mode, b200s_server* srv, int dtype, const void* const* src, void* const* dst, const int32_t* lens,
           int pool, double rate, double duration_s, int32_t window, uint64_t seed, double max_lag_s,
           lg_result* out) {
    *out = lg_result{};
    out->offered_req_per_s = rate;
    const bool open = mode == LG_SERVER_OPEN || mode == LG_PLAIN_OPEN;
    const bool server = mode == LG_SERVER_OPEN || mode == LG_SERVER_CLOSED;
    if (pool <= 0 || (server && !srv) || (open && rate <= 0) || (!open && window <= 0)) return 1;
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(open ? rate : 1.0);
    const int64_t dur_ns = int64_t(duration_s * 1e9);
    const int64_t lag_limit = int64_t(max_lag_s * 1e9);

    if (server) {
        b200s_server_stats st;
        b200s_server_stats_get(srv, &st, 1);  // reset
        std::vector<uint64_t> ring(size_t(std::max(window, 1)));
        const int64_t t0 = now_ns() + 1000000;
        double t_next = double(t0);
        int64_t i = 0, done = 0, keys = 0;
        int64_t max_lag = 0;
        for (;;) {
            int64_t t_arr;
            if (open) {
                t_arr = int64_t(t_next);
                if (t_arr - t0 > dur_ns) break;
                while (now_ns() < t_arr) {
                }
                const int64_t lag = now_ns() - t_arr;
                max_lag = std::max(max_lag, lag);
                if (lag > lag_limit) {
                    out->overloaded = 1;
                    break;
                }
                t_next += gap(rng) * 1e9;
            } else {
                if (now_ns() - t0 > dur_ns) break;
                if (i - done >= window) {
                    b200s_status r;
                    const b200s_status w = b200s_server_wait(srv, ring[size_t(done % window)], -1, &r);
                    if (w != B200S_OK) return int(w);
                    ++done;
                    continue;
                }
                t_arr = now_ns();
            }
            const int k = int(i % pool);
            uint64_t ticket = 0;
            const b200s_status s =
                b200s_server_submit_arrived(srv, src[k], dst[k], lens[k], B200S_MEM_DEVICE, t_arr, &ticket);
            if (s == B200S_ERR_BUSY) {
                ++out->rejected;
                if (!open) std::this_thread::yield();
                continue;
            }
            if (s != B200S_OK) return int(s);
            if (!open) ring[size_t(i % window)] = ticket;
            keys += lens[k];
            ++i;
        }
        b200s_server_drain(srv, -1);
        b200s_server_stats_get(srv, &st, 0);
        out->submitted = i;
        out->completed = st.completed;
        out->rejected += st.rejected;
        out->batches = st.batches;
        out->peak_arena_bytes = st.peak_arena_bytes;
        out->p50_us = st.p50_us;
        out->p99_us = st.p99_us;
        out->p999_us = st.p999_us;
        out->max_us = st.max_us;
        out->mean_us = st.mean_us;
        out->span_s = st.span_s;
        out->keys_per_s = st.span_s > 0 ? double(st.keys_completed) / st.span_s : 0;
        out->req_per_s = st.span_s > 0 ? double(st.completed) / st.span_s : 0;
        out->max_lag_us = double(max_lag) * 1e-3;
        out->mean_batch = st.mean_batch_requests;
        return st.failed ? 3 : 0;
    }

    // plain per-request launches on one stream; a completion thread polls
    // one event per request in order
    cudaStream_t stream;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return 1000;
    const int kEvents = 4096;
    std::vector<cudaEvent_t> ev(kEvents);
    for (auto& e : ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return 1001;
    const size_t cap = open ? size_t(rate * duration_s * 1.05 + 4096) : size_t(1) << 24;
    std::vector<int64_t> t_arr(cap), lat(cap);
    std::vector<int32_t> nkeys(cap);
    std::atomic<int64_t> submitted{0}, completed{0};
    std::atomic<int> stop{0}, cuda_err{0};
    std::thread poller([&] {
        int64_t j = 0;
        for (;;) {
            const int64_t s = submitted.load(std::memory_order_acquire);
            if (j >= s) {
                if (stop.load(std::memory_order_acquire) && j >= submitted.load()) break;
                std::this_thread::yield();
                continue;
            }
            const cudaError_t q = cudaEventQuery(ev[size_t(j % kEvents)]);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) {
                cuda_err.store(int(q));
                stop.store(1);
                break;
            }
            lat[size_t(j)] = now_ns() - t_arr[size_t(j)];
            ++j;
            completed.store(j, std::memory_order_release);
        }
    });
    const int64_t t0 = now_ns() + 1000000;
    double t_next = double(t0);
    int64_t i = 0, max_lag = 0;
    int rc = 0;
    for (; size_t(i) < cap; ++i) {
        int64_t ta;
        if (open) {
            ta = int64_t(t_next);
            if (ta - t0 > dur_ns) break;
            while (now_ns() < ta) {
            }
            t_next += gap(rng) * 1e9;
        } else {
            if (now_ns() - t0 > dur_ns) break;
            while (i - completed.load(std::memory_order_acquire) >= window) {
            }
            ta = now_ns();
        }
        // an event is reused only after its request completed
        while (i - completed.load(std::memory_order_acquire) >= kEvents) {
        }
        const int64_t lag = now_ns() - ta;
        max_lag = std::max(max_lag, lag);
        if (open && lag > lag_limit) {
            out->overloaded = 1;
            break;
        }
        const int k = int(i % pool);
        t_arr[size_t(i)] = ta;
        nkeys[size_t(i)] = lens[k];
        const b200s_status s = b200s_sort_packed(b200s_dtype(dtype), src[k], dst[k], lens[k], 1, 0, nullptr, stream);
        if (s != B200S_OK) {
            rc = int(s);
            break;
        }
        if (cudaEventRecord(ev[size_t(i % kEvents)], stream) != cudaSuccess) {
            rc = 1002;
            break;
        }
        submitted.store(i + 1, std::memory_order_release);
        if (cuda_err.load()) break;
    }
    stop.store(1, std::memory_order_release);
    poller.join();
    cudaStreamSynchronize(stream);
    const int64_t n = completed.load();
    int64_t keys = 0, t_last = t0;
    for (int64_t j = 0; j < n; ++j) {
        keys += nkeys[size_t(j)];
        t_last = std::max(t_last, t_arr[size_t(j)] + lat[size_t(j)]);
    }
    std::vector<int64_t> l(lat.begin(), lat.begin() + n);
    const Percentiles p = percentiles(l);
    out->submitted = i;
    out->completed = n;
    out->batches = n;
    out->p50_us = p.p50;
    out->p99_us = p.p99;
    out->p999_us = p.p999;
    out->max_us = p.max;
    out->mean_us = p.mean;
    out->span_s = n ? double(t_last - t_arr[0]) * 1e-9 : 0;
    out->keys_per_s = out->span_s > 0 ? double(keys) / out->span_s : 0;
    out->req_per_s = out->span_s > 0 ? double(n) / out->span_s : 0;
    out->max_lag_us = double(max_lag) * 1e-3;
    out->mean_batch = 1;
    for (auto& e : ev) cudaEventDestroy(e);
    cudaStreamDestroy(stream);
    if (cuda_err.load()) return 1000 + cuda_err.load();
    return rc;
}

}  // extern "C"
