// Continuous-batching request scheduler of the b200sort server.
//
// This header holds the serving policy and no CUDA: requests are queued by
// any host thread; one worker thread admits them into batches as device
// slots and arena memory free up, hands each batch to a Backend, polls the
// batches in flight, completes their requests and records latencies.  The
// CUDA backend lives in server.cu; the host tests instantiate the same core
// with a fake backend, so admission, the memory budget, cancellation, error
// propagation and the latency statistics are tested without a GPU.
//
// The reference has no serving path; its nearest relative is the stream pool
// that runs oversized partitions concurrently (cusort.hpp:114-122,
// 2633-2652), which schedules one known batch, not arriving requests.
//
// Backend contract (B is a class with these members):
//   int      slots() const                  batches that may be in flight at once
//   int64_t  arena_elems() const            device arena capacity in elements (the budget)
//   int      elem_bytes() const             bytes per element
//   int      align_elems() const            request starts are multiples of this
//   int32_t  max_length() const             longest request
//   b200s_status launch(int slot, const Item* items, int count, int64_t region_elem,
//                       int64_t region_elems, std::string* err)
//                                           stage, sort and return the batch (async)
//   int      query(int slot, std::string* err)  0 running, 1 done, -1 failed
#pragma once
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "b200sort.h"

namespace b200s {
namespace serving {

inline int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// One request, in a fixed table slot (ticket % capacity).
struct Request {
    uint64_t ticket = 0;
    const void* src = nullptr;
    void* dst = nullptr;
    int32_t n = 0;
    uint32_t mem = 0;
    int64_t t_submit = 0;
    int64_t t_done = 0;
    std::atomic<int> state{B200S_REQ_FREE};
    int status = B200S_OK;
};

// What the backend receives for each request of a batch.
struct Item {
    Request* req;
    int64_t arena_elem;  // first element of the request's arena slot
    int32_t n_pad;       // slot length: n rounded up to align_elems()
};

// Arena space is handed out as one contiguous region per batch, in a ring,
// and released in admission order.  Positions are in elements.  Free space
// is [head, cap) + [0, tail) when head >= tail, else [head, tail); a region
// that would not fit before the end starts again at 0 and owns the skipped
// end.
class RingArena {
public:
    struct Region {
        int64_t begin, end, skipped;
    };
    explicit RingArena(int64_t capacity) : cap_(capacity) {}
    int64_t capacity() const { return cap_; }
    int64_t used() const { return used_; }

    // Extend the open region by `elems` (a new region when new_region).
    // Returns the element position, or -1 when that space is not free.
    int64_t grow(int64_t elems, bool new_region) {
        if (elems <= 0 || elems > cap_) return -1;
        if (used_ == 0) head_ = tail_ = 0;
        if (used_ == cap_) return -1;
        if (head_ >= tail_) {
            if (head_ + elems <= cap_) return take(elems);
            if (new_region && elems <= tail_) {
                skipped_ = cap_ - head_;
                used_ += skipped_;
                head_ = 0;
                return take(elems);
            }
            return -1;
        }
        if (head_ + elems <= tail_) return take(elems);
        return -1;
    }
    // Close the open region that started at `begin`.
    Region close(int64_t begin) {
        Region r{begin, head_, skipped_};
        skipped_ = 0;
        return r;
    }
    // Release the oldest live region.
    void release(const Region& r) {
        used_ -= (r.end - r.begin) + r.skipped;
        tail_ = r.end;
        if (used_ == 0) head_ = tail_ = 0;
    }

private:
    int64_t take(int64_t elems) {
        const int64_t at = head_;
        head_ += elems;  // may reach cap_: the next region wraps
        used_ += elems;
        return at;
    }
    int64_t cap_;
    int64_t head_ = 0, tail_ = 0, used_ = 0, skipped_ = 0;
};

struct Limits {
    int32_t max_batch_arrays = 4096;  // requests per batch
    int64_t max_batch_elems = int64_t(1) << 28;
    int64_t max_queue = 1 << 16;      // request table capacity
    size_t max_samples = size_t(1) << 24;  // latency samples kept (the most recent)
};

template <class B>
class ServerCore {
public:
    ServerCore(std::unique_ptr<B> backend, const Limits& lim)
        : be_(std::move(backend)), lim_(lim), arena_(be_->arena_elems()), table_(size_t(lim.max_queue)),
          slot_busy_(size_t(be_->slots()), 0) {
        worker_ = std::thread([this] { loop(); });
    }
    ~ServerCore() { shutdown(); }

    B& backend() { return *be_; }

    // Stop admitting: queued requests are cancelled, admitted ones finish.
    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stopping_ = true;
        }
        cv_work_.notify_all();
        std::lock_guard<std::mutex> j(join_mu_);
        if (worker_.joinable()) worker_.join();
    }

    // t_arrival: when the request arrived (now_ns() timeline), 0 for now;
    // latencies run from it.
    b200s_status submit(const void* src, void* dst, int32_t n, uint32_t mem, uint64_t* ticket,
                        std::string* err, int64_t t_arrival = 0) {
        if (!ticket) return fail(err, B200S_ERR_INVALID_ARGUMENT, "null ticket pointer");
        if (n < 0) return fail(err, B200S_ERR_INVALID_ARGUMENT, "negative length");
        if (mem > B200S_MEM_HOST) return fail(err, B200S_ERR_INVALID_ARGUMENT, "unknown memory kind");
        if (n > 0 && (!src || !dst)) return fail(err, B200S_ERR_INVALID_ARGUMENT, "null buffer");
        if (n > be_->max_length())
            return fail(err, B200S_ERR_UNSUPPORTED,
                        "request of " + std::to_string(n) + " elements exceeds the longest sortable array (" +
                            std::to_string(be_->max_length()) + ")");
        const int64_t slot_elems = pad(n);
        if (slot_elems > arena_.capacity() || slot_elems > lim_.max_batch_elems) {
            rejected_.fetch_add(1, std::memory_order_relaxed);
            return fail(err, B200S_ERR_BUDGET,
                        "request of " + std::to_string(slot_elems * be_->elem_bytes()) +
                            " bytes exceeds the server's device-memory budget of " +
                            std::to_string(arena_.capacity() * be_->elem_bytes()) + " bytes");
        }
        std::unique_lock<std::mutex> lk(mu_);
        if (stopping_) return fail(err, B200S_ERR_INVALID_ARGUMENT, "server is shutting down");
        const uint64_t t = next_ticket_;
        Request& r = table_[size_t(t % table_.size())];
        const int st = r.state.load(std::memory_order_acquire);
        if (st == B200S_REQ_QUEUED || st == B200S_REQ_RUNNING) {
            rejected_.fetch_add(1, std::memory_order_relaxed);
            return fail(err, B200S_ERR_BUSY,
                        "request table full (" + std::to_string(table_.size()) + " requests pending)");
        }
        ++next_ticket_;
        r.ticket = t;
        r.src = src;
        r.dst = dst;
        r.n = n;
        r.mem = mem;
        r.status = B200S_OK;
        r.t_submit = t_arrival > 0 ? t_arrival : now_ns();
        r.t_done = 0;
        ++submitted_;
        if (first_submit_ == 0 || r.t_submit < first_submit_) first_submit_ = r.t_submit;
        *ticket = t;
        if (n == 0) {
            r.t_done = std::max(r.t_submit, now_ns());
            r.state.store(B200S_REQ_DONE, std::memory_order_release);
            record_done_locked(r);
            lk.unlock();
            cv_done_.notify_all();
            return B200S_OK;
        }
        r.state.store(B200S_REQ_QUEUED, std::memory_order_release);
        queue_.push_back(&r);
        lk.unlock();
        cv_work_.notify_one();
        return B200S_OK;
    }

    // State of a ticket; B200S_REQ_FREE for tickets never issued or recycled.
    int state_of(uint64_t ticket, int* status) {
        std::lock_guard<std::mutex> lk(mu_);
        if (ticket >= next_ticket_) return B200S_REQ_FREE;
        const Request& r = table_[size_t(ticket % table_.size())];
        if (r.ticket != ticket) return B200S_REQ_FREE;
        if (status) *status = r.status;
        return r.state.load(std::memory_order_acquire);
    }

    b200s_status wait(uint64_t ticket, int64_t timeout_us, b200s_status* result, std::string* err) {
        std::unique_lock<std::mutex> lk(mu_);
        if (ticket >= next_ticket_) return fail(err, B200S_ERR_INVALID_ARGUMENT, "unknown ticket");
        const Request& r = table_[size_t(ticket % table_.size())];
        auto finished = [&] {
            if (r.ticket != ticket) return true;  // recycled: it finished long ago
            const int s = r.state.load(std::memory_order_acquire);
            return s == B200S_REQ_DONE || s == B200S_REQ_FAILED || s == B200S_REQ_CANCELLED;
        };
        if (timeout_us < 0) {
            cv_done_.wait(lk, finished);
        } else if (!cv_done_.wait_for(lk, std::chrono::microseconds(timeout_us), finished)) {
            return fail(err, B200S_ERR_TIMEOUT, "request still pending");
        }
        if (r.ticket != ticket) return fail(err, B200S_ERR_INVALID_ARGUMENT, "ticket recycled");
        if (result) *result = b200s_status(r.status);
        return B200S_OK;
    }

    // Cancel a request that is still queued (admitted requests run to the end).
    b200s_status cancel(uint64_t ticket, std::string* err) {
        std::unique_lock<std::mutex> lk(mu_);
        if (ticket >= next_ticket_) return fail(err, B200S_ERR_INVALID_ARGUMENT, "unknown ticket");
        Request& r = table_[size_t(ticket % table_.size())];
        if (r.ticket != ticket || r.state.load() != B200S_REQ_QUEUED)
            return fail(err, B200S_ERR_INVALID_ARGUMENT, "request is not queued");
        for (auto it = queue_.begin(); it != queue_.end(); ++it)
            if (*it == &r) {
                queue_.erase(it);
                break;
            }
        r.status = B200S_ERR_CANCELLED;
        r.t_done = now_ns();
        r.state.store(B200S_REQ_CANCELLED, std::memory_order_release);
        ++cancelled_;
        lk.unlock();
        cv_done_.notify_all();
        return B200S_OK;
    }

    b200s_status drain(int64_t timeout_us, std::string* err) {
        std::unique_lock<std::mutex> lk(mu_);
        auto idle = [&] { return queue_.empty() && inflight_ == 0; };
        if (timeout_us < 0) {
            cv_done_.wait(lk, idle);
        } else if (!cv_done_.wait_for(lk, std::chrono::microseconds(timeout_us), idle)) {
            return fail(err, B200S_ERR_TIMEOUT, "requests still pending");
        }
        return B200S_OK;
    }

    void stats(b200s_server_stats* out, bool reset) {
        std::lock_guard<std::mutex> lk(mu_);
        *out = b200s_server_stats{};
        out->submitted = submitted_;
        out->completed = completed_;
        out->failed = failed_;
        out->cancelled = cancelled_;
        out->rejected = rejected_.load();
        out->batches = batches_;
        out->keys_completed = keys_done_;
        out->queued = int64_t(queue_.size());
        out->inflight_batches = inflight_;
        out->peak_arena_bytes = peak_arena_ * be_->elem_bytes();
        out->arena_bytes = arena_.capacity() * be_->elem_bytes();
        out->max_batch_requests = max_batch_seen_;
        out->mean_batch_requests = batches_ ? double(batched_reqs_) / double(batches_) : 0.0;
        out->span_s = (first_submit_ && last_done_ > first_submit_) ? double(last_done_ - first_submit_) * 1e-9 : 0.0;
        if (!lat_.empty()) {
            std::vector<int64_t> v(lat_);
            auto pct = [&](double q) {
                const size_t k = size_t(q * double(v.size() - 1) + 0.5);
                std::nth_element(v.begin(), v.begin() + long(k), v.end());
                return double(v[k]) * 1e-3;
            };
            out->p50_us = pct(0.50);
            out->p99_us = pct(0.99);
            out->p999_us = pct(0.999);
            out->max_us = double(*std::max_element(v.begin(), v.end())) * 1e-3;
            double s = 0;
            for (int64_t x : v) s += double(x);
            out->mean_us = s / double(v.size()) * 1e-3;
        }
        if (reset) {
            submitted_ = completed_ = failed_ = cancelled_ = batches_ = keys_done_ = 0;
            batched_reqs_ = max_batch_seen_ = 0;
            rejected_.store(0);
            peak_arena_ = arena_.used();
            first_submit_ = last_done_ = 0;
            lat_.clear();
            lat_next_ = 0;
        }
    }

    std::string last_error() {
        std::lock_guard<std::mutex> lk(mu_);
        return last_error_;
    }

private:
    struct Batch {
        int slot;
        std::vector<Request*> reqs;
        RingArena::Region region;
        bool done = false;
    };

    static b200s_status fail(std::string* err, b200s_status s, const std::string& m) {
        if (err) *err = m;
        return s;
    }

    int64_t pad(int32_t n) const {
        const int64_t a = be_->align_elems();
        return (int64_t(n) + a - 1) / a * a;
    }

    // mu_ held.
    void record_done_locked(const Request& r) {
        if (r.state.load() == B200S_REQ_DONE) {
            ++completed_;
            keys_done_ += r.n;
            const int64_t lat = r.t_done - r.t_submit;
            if (lat_.size() < lim_.max_samples) {
                lat_.push_back(lat);
            } else {
                lat_[lat_next_] = lat;
                lat_next_ = (lat_next_ + 1) % lat_.size();
            }
        } else {
            ++failed_;
        }
        last_done_ = std::max(last_done_, r.t_done);
    }

    // mu_ held: finish the requests of a batch.
    void finish_locked(Batch& b, int outcome, b200s_status fail_status, const std::string& err) {
        const int64_t t = now_ns();
        for (Request* r : b.reqs) {
            r->t_done = t;
            r->status = outcome > 0 ? B200S_OK : fail_status;
            r->state.store(outcome > 0 ? B200S_REQ_DONE : B200S_REQ_FAILED, std::memory_order_release);
            record_done_locked(*r);
        }
        if (outcome <= 0) last_error_ = err;
        b.done = true;
        slot_busy_[size_t(b.slot)] = 0;
        --inflight_;
    }

    // mu_ held: give back the arena regions of the oldest finished batches.
    void release_locked() {
        while (!inflight_list_.empty() && inflight_list_.front().done) {
            arena_.release(inflight_list_.front().region);
            inflight_list_.pop_front();
        }
    }

    // Retire finished batches; returns true if anything changed.
    bool retire() {
        bool changed = false;
        for (Batch& b : inflight_list_) {
            if (b.done) continue;
            std::string err;
            const int q = be_->query(b.slot, &err);
            if (q == 0) continue;
            std::lock_guard<std::mutex> lk(mu_);
            finish_locked(b, q, B200S_ERR_CUDA, err);
            changed = true;
        }
        if (changed) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                release_locked();
            }
            cv_done_.notify_all();
        }
        return changed;
    }

    int free_slot() const {
        for (size_t i = 0; i < slot_busy_.size(); ++i)
            if (!slot_busy_[i]) return int(i);
        return -1;
    }

    // Admit queued requests into batches while slots and arena space allow.
    bool admit() {
        bool changed = false;
        for (;;) {
            const int slot = free_slot();
            if (slot < 0) return changed;
            Batch b;
            b.slot = slot;
            items_.clear();
            int64_t begin = -1, elems = 0;
            {
                std::lock_guard<std::mutex> lk(mu_);
                while (!queue_.empty() && int32_t(b.reqs.size()) < lim_.max_batch_arrays) {
                    Request* r = queue_.front();
                    const int64_t len = pad(r->n);
                    if (elems + len > lim_.max_batch_elems) break;
                    const int64_t at = arena_.grow(len, b.reqs.empty());
                    if (at < 0) break;  // wait for memory to free up
                    if (b.reqs.empty()) begin = at;
                    queue_.pop_front();
                    r->state.store(B200S_REQ_RUNNING, std::memory_order_release);
                    b.reqs.push_back(r);
                    items_.push_back(Item{r, at, int32_t(len)});
                    elems += len;
                }
                if (b.reqs.empty()) return changed;
                b.region = arena_.close(begin);
                peak_arena_ = std::max(peak_arena_, arena_.used());
                ++inflight_;
                ++batches_;
                batched_reqs_ += int64_t(b.reqs.size());
                max_batch_seen_ = std::max<int64_t>(max_batch_seen_, int64_t(b.reqs.size()));
                slot_busy_[size_t(slot)] = 1;
            }
            std::string err;
            const b200s_status st = be_->launch(slot, items_.data(), int(items_.size()), begin, elems, &err);
            {
                std::lock_guard<std::mutex> lk(mu_);
                inflight_list_.push_back(std::move(b));
                if (st != B200S_OK) {
                    finish_locked(inflight_list_.back(), -1, st, err);
                    release_locked();
                }
            }
            if (st != B200S_OK) cv_done_.notify_all();
            changed = true;
        }
    }

    void loop() {
        int idle_spins = 0;
        int64_t last_active = now_ns();
        for (;;) {
            bool progressed = retire();
            progressed = admit() || progressed;
            std::unique_lock<std::mutex> lk(mu_);
            if (stopping_) {
                // Requests never admitted are cancelled; admitted ones finish.
                const bool had = !queue_.empty();
                while (!queue_.empty()) {
                    Request* r = queue_.front();
                    queue_.pop_front();
                    r->status = B200S_ERR_CANCELLED;
                    r->t_done = now_ns();
                    r->state.store(B200S_REQ_CANCELLED, std::memory_order_release);
                    ++cancelled_;
                }
                if (had) cv_done_.notify_all();
                if (inflight_ == 0) return;
            }
            if (progressed) {
                idle_spins = 0;
                last_active = now_ns();
                continue;
            }
            if (inflight_ == 0 && queue_.empty()) {
                // Idle: keep polling for a short while (a request arriving
                // soon after another is admitted without a thread wake-up),
                // then sleep until a submission.
                if (now_ns() - last_active < kIdleSpinNs) {
                    lk.unlock();
                    std::this_thread::yield();
                    continue;
                }
                cv_work_.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
            lk.unlock();
            // Batches are in flight: poll them.
            if (++idle_spins > 64) std::this_thread::yield();
        }
    }

    static constexpr int64_t kIdleSpinNs = 200000;

    std::unique_ptr<B> be_;
    Limits lim_;
    RingArena arena_;
    std::vector<Request> table_;
    std::vector<char> slot_busy_;
    std::deque<Batch> inflight_list_;
    std::vector<Item> items_;  // worker thread only

    std::mutex mu_;      // everything below, and the arena, slots and in-flight list
    std::mutex join_mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<Request*> queue_;
    bool stopping_ = false;
    uint64_t next_ticket_ = 0;
    int inflight_ = 0;
    int64_t submitted_ = 0, completed_ = 0, failed_ = 0, cancelled_ = 0, batches_ = 0, keys_done_ = 0;
    int64_t batched_reqs_ = 0, max_batch_seen_ = 0, peak_arena_ = 0;
    int64_t first_submit_ = 0, last_done_ = 0;
    std::atomic<int64_t> rejected_{0};
    std::vector<int64_t> lat_;
    size_t lat_next_ = 0;
    std::string last_error_;
    std::thread worker_;
};

}  // namespace serving
}  // namespace b200s
