// Build-time driver for the reference's GPU kernels (TEST INFRASTRUCTURE).
//
// Compiled by oracle/Makefile against the unmodified reference headers for
// sm_100a into oracle/_ref/libref_gpu.so.  It wraps the reference's device
// entry points in the same batched form its bench uses (segment = data +
// blockIdx.x * n, in place: bench.cu:355-393) so that tests can compare the
// new kernels' outputs with the reference's own outputs on a B200, and time
// the reference V6 kernel on the same inputs.
//
// REF_TYPE selects the element type of this translation unit (0 = int,
// 1 = IntAndData); the Makefile builds one object per type.
#include <cstdint>

#include "cusort.hpp"
#include "cusort_experiments.hpp"
#include "cusort_v6.hpp"
#include "intanddata.hpp"

#if REF_TYPE == 0
using Elem = int;
#define REF_SUFFIX(name) name##_int
constexpr unsigned kMaxWorking = 4096;
#else
using Elem = IntAndData;
#define REF_SUFFIX(name) name##_rec
constexpr unsigned kMaxWorking = 2048;
#endif

namespace {

template <unsigned W, unsigned Th, bool Sorted, bool Shared, bool Async>
__global__ void v6_batched(Elem* data, int n) {
    Elem* seg = data + size_t(blockIdx.x) * n;
    cusort_v6::Sort<Elem, W, Th, Sorted, Shared, Async>(seg, seg, n);
}

template <bool Sorted, bool Shared>
__global__ void warp_batched(Elem* data, int n) {
    Elem* seg = data + size_t(blockIdx.x) * n;
    Sort_1Warp_SM_le32_d<Elem, Sorted, Shared>(seg, seg, n);
}

template <bool Sorted, bool Shared, bool Async>
__global__ void v3_batched(Elem* data, int n, int working) {
    Elem* seg = data + size_t(blockIdx.x) * n;
    if constexpr (Async) Sort_1Block_async_gt32_d_extsm_v3<Elem, Sorted, Shared>(seg, seg, n, working);
    else Sort_1Block_gt32_d_extsm_v3<Elem, Sorted, Shared>(seg, seg, n, working);
}

template <bool Sorted, bool Shared, bool Async>
__global__ void v4_batched(Elem* data, int n, unsigned working) {
    Elem* seg = data + size_t(blockIdx.x) * n;
    cusort_experiment::Sort<Elem, Sorted, Shared, Async>(seg, seg, n, working);
}

int launch_status() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

template <unsigned W, unsigned Th, bool Sorted, bool Shared, bool Async>
int run_v6(Elem* d, int n, int arrays, cudaStream_t st) {
    auto k = v6_batched<W, Th, Sorted, Shared, Async>;
    const size_t bytes = 2 * size_t(W) * sizeof(Elem);
    if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    k<<<arrays, Th, bytes, st>>>(d, n);
    return launch_status();
}

template <unsigned W, unsigned Th>
int pick_flags(int sorted, int shared, int async, Elem* d, int n, int arrays, cudaStream_t st) {
    const int key = (sorted ? 4 : 0) | (shared ? 2 : 0) | (async ? 1 : 0);
    switch (key) {
        case 0: return run_v6<W, Th, false, false, false>(d, n, arrays, st);
        case 1: return run_v6<W, Th, false, false, true>(d, n, arrays, st);
        case 2: return run_v6<W, Th, false, true, false>(d, n, arrays, st);
        case 3: return run_v6<W, Th, false, true, true>(d, n, arrays, st);
        case 4: return run_v6<W, Th, true, false, false>(d, n, arrays, st);
        default: return 1;
    }
}

template <unsigned W, unsigned Th>
int try_threads(int threads, int sorted, int shared, int async, Elem* d, int n, int arrays,
                cudaStream_t st) {
    if constexpr (Th <= 1024) {
        if constexpr (Th <= W && W / Th <= 16) {
            if (unsigned(threads) == Th) return pick_flags<W, Th>(sorted, shared, async, d, n, arrays, st);
        }
        return try_threads<W, Th * 2>(threads, sorted, shared, async, d, n, arrays, st);
    }
    return 1;
}

template <unsigned W>
int try_working(int working, int threads, int sorted, int shared, int async, Elem* d, int n,
                int arrays, cudaStream_t st) {
    if constexpr (W <= kMaxWorking) {
        if (unsigned(working) == W) return try_threads<W, 32>(threads, sorted, shared, async, d, n, arrays, st);
        return try_working<W * 2>(working, threads, sorted, shared, async, d, n, arrays, st);
    }
    return 1;
}

}  // namespace

extern "C" {

// Reference V6 (cusort_v6.hpp) over a packed batch, in place.  working must
// be the next power of two >= max(32, n), as bench.cu:524 computes it.
// Returns 0 on success, 1 for an uncompiled configuration, 2 on a CUDA error.
int REF_SUFFIX(ref_v6)(void* d, int n, int arrays, int working, int threads, int sorted, int shared,
                       int async, void* stream) {
    return try_working<32>(working, threads, sorted, shared, async, static_cast<Elem*>(d), n, arrays,
                           static_cast<cudaStream_t>(stream));
}

// Reference warp sort for n <= 32 (cusort.hpp:574-596), 32 threads per array.
int REF_SUFFIX(ref_warp)(void* d, int n, int arrays, int sorted, int shared, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Elem* p = static_cast<Elem*>(d);
    if (n > 32) return 1;
    if (sorted && shared) warp_batched<true, true><<<arrays, 32, 0, st>>>(p, n);
    else if (sorted) warp_batched<true, false><<<arrays, 32, 0, st>>>(p, n);
    else if (shared) warp_batched<false, true><<<arrays, 32, 0, st>>>(p, n);
    else warp_batched<false, false><<<arrays, 32, 0, st>>>(p, n);
    return launch_status();
}

// Reference V3 (cusort.hpp:1229-1300): any warp-multiple block, 2W smem.
int REF_SUFFIX(ref_v3)(void* d, int n, int arrays, int working, int threads, int sorted, int shared,
                       int async, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Elem* p = static_cast<Elem*>(d);
    const size_t bytes = 2 * size_t(working) * sizeof(Elem);
    const int key = (sorted ? 4 : 0) | (shared ? 2 : 0) | (async ? 1 : 0);
    switch (key) {
        case 0: v3_batched<false, false, false><<<arrays, threads, bytes, st>>>(p, n, working); break;
        case 1: v3_batched<false, false, true><<<arrays, threads, bytes, st>>>(p, n, working); break;
        case 2: v3_batched<false, true, false><<<arrays, threads, bytes, st>>>(p, n, working); break;
        case 4: v3_batched<true, false, false><<<arrays, threads, bytes, st>>>(p, n, working); break;
        default: return 1;
    }
    return launch_status();
}

// Reference V4 (cusort_experiments.hpp:366-414): runtime working length.
int REF_SUFFIX(ref_v4)(void* d, int n, int arrays, int working, int threads, int sorted, int shared,
                       int async, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Elem* p = static_cast<Elem*>(d);
    const size_t bytes = 2 * size_t(working) * sizeof(Elem);
    const int key = (sorted ? 4 : 0) | (shared ? 2 : 0) | (async ? 1 : 0);
    switch (key) {
        case 0: v4_batched<false, false, false><<<arrays, threads, bytes, st>>>(p, n, unsigned(working)); break;
        case 1: v4_batched<false, false, true><<<arrays, threads, bytes, st>>>(p, n, unsigned(working)); break;
        case 2: v4_batched<false, true, false><<<arrays, threads, bytes, st>>>(p, n, unsigned(working)); break;
        case 4: v4_batched<true, false, false><<<arrays, threads, bytes, st>>>(p, n, unsigned(working)); break;
        default: return 1;
    }
    return launch_status();
}

}  // extern "C"
