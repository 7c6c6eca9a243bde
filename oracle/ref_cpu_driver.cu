// Build-time driver for the reference's own CPU path (TEST INFRASTRUCTURE).
//
// Compiled by oracle/Makefile against the unmodified reference headers into
// oracle/_ref/libref_cpu.so.  It exposes, over plain pointers, exactly what
// the reference does on the host to build its expected output: one std::sort
// per array with the reference's element type and ordering (bench.cu:300-301,
// IntAndData::operator< from intanddata.hpp:20-22).  Arrays are spread over
// std::thread workers in static contiguous chunks.
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "cusort.hpp"
#include "intanddata.hpp"

namespace {
template <class T>
void sort_arrays(T* data, long long n, long long arrays, int threads) {
    auto work = [&](long long lo, long long hi) {
        for (long long a = lo; a < hi; ++a) std::sort(data + a * n, data + (a + 1) * n);
    };
    if (threads <= 1) {
        work(0, arrays);
        return;
    }
    std::vector<std::thread> pool;
    const long long chunk = (arrays + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const long long lo = t * chunk, hi = std::min(arrays, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back(work, lo, hi);
    }
    for (auto& th : pool) th.join();
}

template <class T>
void sort_ragged(T* data, const long long* off, long long arrays, int threads) {
    auto work = [&](long long lo, long long hi) {
        for (long long a = lo; a < hi; ++a) std::sort(data + off[a], data + off[a + 1]);
    };
    if (threads <= 1) {
        work(0, arrays);
        return;
    }
    // Interleaved chunks of 64 arrays balance long and short arrays.
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (long long lo = 64LL * t; lo < arrays; lo += 64LL * threads) work(lo, std::min(arrays, lo + 64));
        });
    for (auto& th : pool) th.join();
}
}  // namespace

extern "C" {
// Ragged batch (CSR offsets, arrays + 1 entries), in place.
int ref_cpu_sort_ragged(int type, void* data, const long long* off, long long arrays, int threads) {
    if (type == 0) sort_ragged(static_cast<int*>(data), off, arrays, threads);
    else if (type == 1) sort_ragged(static_cast<IntAndData*>(data), off, arrays, threads);
    else return 1;
    return 0;
}

// type 0: int keys, type 1: IntAndData records.  Sorts in place.
int ref_cpu_sort(int type, void* data, long long n, long long arrays, int threads) {
    if (type == 0) sort_arrays(static_cast<int*>(data), n, arrays, threads);
    else if (type == 1) sort_arrays(static_cast<IntAndData*>(data), n, arrays, threads);
    else return 1;
    return 0;
}
}
