// Test double for the b200sort server: the real scheduler (serving_core.hpp)
// driven by a fake device that stages, sorts and returns batches on host
// threads, with injectable delays and failures.  Built by
// tests/test_serving_core.py with g++; never part of the library.
//
// The fake device also checks the scheduler's promises: every batch region
// lies inside the arena, a batch's requests are back to back from the region
// start, and no two batches in flight share arena elements.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "serving_core.hpp"

using b200s::serving::Item;
using b200s::serving::Limits;
using b200s::serving::RingArena;
using b200s::serving::ServerCore;

namespace {

thread_local std::string g_err;

class FakeBackend {
public:
    FakeBackend(int eb, int64_t budget, int slots, int32_t max_len, int delay_us)
        : eb_(eb), align_(16 / eb), arena_elems_(budget / 16 * (16 / eb)), max_len_(max_len),
          delay_us_(delay_us), arena_(size_t(arena_elems_) * size_t(eb)), jobs_(size_t(slots)) {
        for (auto& j : jobs_) j = std::make_unique<Job>();
    }
    ~FakeBackend() {
        for (auto& j : jobs_)
            if (j->th.joinable()) j->th.join();
    }
    int slots() const { return int(jobs_.size()); }
    int64_t arena_elems() const { return arena_elems_; }
    int elem_bytes() const { return eb_; }
    int align_elems() const { return align_; }
    int32_t max_length() const { return max_len_; }

    b200s_status launch(int slot, const Item* items, int count, int64_t region, int64_t elems, std::string* err) {
        Job& j = *jobs_[size_t(slot)];
        if (j.th.joinable()) j.th.join();
        if (fail_launch_.exchange(0)) {
            *err = "injected launch failure";
            return B200S_ERR_CUDA;
        }
        // scheduler invariants
        int64_t at = region;
        for (int i = 0; i < count; ++i) {
            if (items[i].arena_elem != at || items[i].n_pad % align_ || items[i].n_pad < items[i].req->n)
                ++violations_;
            at += items[i].n_pad;
        }
        if (at != region + elems || region < 0 || region + elems > arena_elems_) ++violations_;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (const auto& kv : live_)
                if (kv.first != slot && region < kv.second.second && kv.second.first < region + elems) ++violations_;
            live_[slot] = {region, region + elems};
        }
        std::vector<Item> copy(items, items + count);
        const bool fail = fail_complete_.exchange(0) != 0;
        const int delay = delay_us_.load();
        j.state.store(0);
        j.th = std::thread([this, &j, copy, fail, delay, slot] {
            if (delay) std::this_thread::sleep_for(std::chrono::microseconds(delay));
            for (const Item& it : copy) {
                char* s = arena_.data() + size_t(it.arena_elem) * size_t(eb_);
                std::memcpy(s, it.req->src, size_t(it.req->n) * size_t(eb_));
                std::vector<std::vector<char>> rec(size_t(it.req->n));
                for (int k = 0; k < it.req->n; ++k) rec[size_t(k)].assign(s + k * eb_, s + (k + 1) * eb_);
                std::stable_sort(rec.begin(), rec.end(), [](const std::vector<char>& a, const std::vector<char>& b) {
                    int32_t ka, kb;
                    std::memcpy(&ka, a.data(), 4);
                    std::memcpy(&kb, b.data(), 4);
                    return ka < kb;
                });
                for (int k = 0; k < it.req->n; ++k)
                    std::memcpy(static_cast<char*>(it.req->dst) + size_t(k) * size_t(eb_), rec[size_t(k)].data(),
                                size_t(eb_));
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                live_.erase(slot);
            }
            j.state.store(fail ? -1 : 1);
        });
        return B200S_OK;
    }

    int query(int slot, std::string* err) {
        const int s = jobs_[size_t(slot)]->state.load();
        if (s < 0) *err = "injected device failure";
        return s;
    }

    std::atomic<int> fail_launch_{0}, fail_complete_{0}, delay_us_{0};
    std::atomic<int64_t> violations_{0};

private:
    struct Job {
        std::thread th;
        std::atomic<int> state{1};
    };
    int eb_, align_;
    int64_t arena_elems_;
    int32_t max_len_;
    std::vector<char> arena_;
    std::vector<std::unique_ptr<Job>> jobs_;
    std::mutex mu_;
    std::map<int, std::pair<int64_t, int64_t>> live_;
};

using Core = ServerCore<FakeBackend>;

}  // namespace

extern "C" {

void* fake_create(int eb, int64_t budget, int slots, int max_batch, int64_t max_queue, int delay_us,
                  int32_t max_len) {
    Limits lim;
    lim.max_batch_arrays = max_batch;
    lim.max_queue = max_queue;
    auto be = std::make_unique<FakeBackend>(eb, budget, slots, max_len, delay_us);
    return new Core(std::move(be), lim);
}

void fake_destroy(void* s) { delete static_cast<Core*>(s); }
void fake_shutdown(void* s) { static_cast<Core*>(s)->shutdown(); }

int fake_submit(void* s, const void* src, void* dst, int32_t n, uint64_t* ticket) {
    return static_cast<Core*>(s)->submit(src, dst, n, B200S_MEM_HOST, ticket, &g_err);
}

int fake_wait(void* s, uint64_t t, int64_t timeout_us, int* result) {
    b200s_status r = B200S_OK;
    const b200s_status st = static_cast<Core*>(s)->wait(t, timeout_us, &r, &g_err);
    *result = r;
    return st;
}

int fake_poll(void* s, uint64_t t) { return static_cast<Core*>(s)->state_of(t, nullptr); }
int fake_cancel(void* s, uint64_t t) { return static_cast<Core*>(s)->cancel(t, &g_err); }
int fake_drain(void* s, int64_t timeout_us) { return static_cast<Core*>(s)->drain(timeout_us, &g_err); }
void fake_stats(void* s, b200s_server_stats* out, int reset) { static_cast<Core*>(s)->stats(out, reset != 0); }

void fake_inject(void* s, int fail_launch, int fail_complete) {
    auto& be = static_cast<Core*>(s)->backend();
    be.fail_launch_.store(fail_launch);
    be.fail_complete_.store(fail_complete);
}
void fake_set_delay(void* s, int delay_us) { static_cast<Core*>(s)->backend().delay_us_.store(delay_us); }
int64_t fake_violations(void* s) { return static_cast<Core*>(s)->backend().violations_.load(); }
const char* fake_last_error() { return g_err.c_str(); }

// Random grow/close/release sequences on the ring arena against a model of
// the live regions; returns the number of broken invariants.
int64_t fake_arena_selftest(uint64_t seed, int iters, int64_t cap) {
    std::mt19937_64 rng(seed);
    RingArena a(cap);
    struct Live {
        RingArena::Region r;
        std::vector<std::pair<int64_t, int64_t>> spans;
    };
    std::vector<Live> live;
    int64_t bad = 0;
    for (int it = 0; it < iters; ++it) {
        if (!live.empty() && (rng() % 3 == 0)) {
            a.release(live.front().r);
            live.erase(live.begin());
        } else {
            Live l;
            int64_t begin = -1;
            const int items = 1 + int(rng() % 5);
            for (int k = 0; k < items; ++k) {
                const int64_t len = 1 + int64_t(rng() % uint64_t(cap / 3 + 1));
                const int64_t at = a.grow(len, k == 0);
                if (at < 0) break;
                if (k == 0) begin = at;
                else if (at != l.spans.back().second) ++bad;  // not contiguous
                if (at < 0 || at + len > cap) ++bad;
                l.spans.push_back({at, at + len});
            }
            if (l.spans.empty()) continue;
            l.r = a.close(begin);
            for (const Live& o : live)
                for (const auto& x : o.spans)
                    for (const auto& y : l.spans)
                        if (x.first < y.second && y.first < x.second) ++bad;  // overlap
            live.push_back(l);
        }
        int64_t sum = 0;
        for (const Live& o : live)
            for (const auto& x : o.spans) sum += x.second - x.first;
        if (a.used() < sum || a.used() > cap) ++bad;
    }
    while (!live.empty()) {
        a.release(live.front().r);
        live.erase(live.begin());
    }
    if (a.used() != 0) ++bad;
    return bad;
}

}  // extern "C"
