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
#include <algorithm>
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

// V1 / V2: one value per thread, the whole array in one block
// (Sort_1Block_gt32_d_extsm, cusort.hpp:751-771; Sort_1Block_gt32_d_extsm_v2,
// cusort.hpp:986-1008), launched as bench.cu:444-456 does.
template <int Variant, bool Sorted, bool Shared>
__global__ void v12_batched(Elem* data, int n) {
    Elem* seg = data + size_t(blockIdx.x) * n;
    if constexpr (Variant == 1) Sort_1Block_gt32_d_extsm<Elem, Sorted, Shared>(seg, n);
    else Sort_1Block_gt32_d_extsm_v2<Elem, Sorted, Shared>(seg, seg, n);
}

int launch_status() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

template <int Variant>
int run_v12(Elem* d, int n, int arrays, int working, int sorted, int shared, cudaStream_t st) {
    const size_t bytes = size_t(working) * sizeof(Elem) * (Variant == 1 ? 1 : 2);
    const int key = (sorted ? 2 : 0) | (shared ? 1 : 0);
    auto k = key == 0 ? v12_batched<Variant, false, false> : key == 1 ? v12_batched<Variant, false, true>
           : key == 2 ? v12_batched<Variant, true, false> : v12_batched<Variant, true, true>;
    if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    k<<<arrays, working, bytes, st>>>(d, n);
    return launch_status();
}

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

// Reference V1 / V2 over a packed batch, in place: working = threads, a power
// of two in [32, 1024] and >= n.  variant 1 or 2.
int REF_SUFFIX(ref_v12)(void* d, int n, int arrays, int variant, int working, int sorted, int shared,
                        void* stream) {
    if (working < 32 || working > 1024 || (working & (working - 1)) || n > working || n < 1) return 1;
    Elem* p = static_cast<Elem*>(d);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return variant == 1 ? run_v12<1>(p, n, arrays, working, sorted, shared, st)
                        : run_v12<2>(p, n, arrays, working, sorted, shared, st);
}

// The reference's partition stage of its large-array sort, as
// HybridSortPartitionedV3 (cusort.hpp:2493-2588) runs it with its default
// parameters (MaxValuesToSort 2048, MaxNbParts 1024, FullSM): pivots from the
// data, per-partition counts and single-value flags, CSR counters, and the
// scatter of d_data into key-range partitions.  Copies the partitioned values
// to d_parts (n elements), the counters to d_counters (nb_parts + 1) and the
// flags to d_uniform (nb_parts); *nb_parts_out receives the partition count
// and *skipped_out 1 when the reference found a single partition and skipped
// the scatter (then d_parts is d_data unchanged and there is one partition).
int REF_SUFFIX(ref_partition_v3)(void* d_data, int n, void* d_parts, int* d_counters, int* d_uniform,
                                 int* nb_parts_out, int* skipped_out, void* stream) {
    constexpr int kMaxValues = 2048, kMaxParts = 1024;
    constexpr bool kFullSM = true;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Elem* data = static_cast<Elem*>(d_data);
    if (n <= 1) return 1;
    CuSortWorkspace<Elem, kMaxParts> ws;
    ws.reserve(size_t(n));
    // the reference's step sequence (cusort.hpp:2514-2573), in its order
    const int candidate = std::min(kMaxParts, std::max(32, 1 + (n - 1) / kMaxValues));
    const int pivot_threads = std::max(32, GreaterPowerOf2EqualOrLarger(candidate));
    if (pivot_threads * 2 <= DefaultNbThreadsPerBlock)
        Sort_core_buildPivots<Elem, kMaxParts, 2, false, kFullSM><<<1, pivot_threads * 2, 0, st>>>(
            data, n, ws.pivots(), candidate);
    else
        Sort_core_buildPivots<Elem, kMaxParts, 1, false, kFullSM><<<1, DefaultNbThreadsPerBlock, 0, st>>>(
            data, n, ws.pivots(), candidate);
    AdaptPartitionCountDevice<Elem, kMaxParts><<<1, 1, 0, st>>>(ws.pivots(), candidate, ws.activeNbParts());
    cudaMemsetAsync(ws.counters(), 0, (candidate + 2) * sizeof(int), st);
    const int all_blocks = (n + DefaultNbThreadsPerBlock - 1) / DefaultNbThreadsPerBlock;
    const int blocks = std::max(1, std::min(all_blocks, ws.persistentBlocks()));
    CountParts_Persistent<Elem, kMaxParts><<<blocks, DefaultNbThreadsPerBlock, 0, st>>>(
        data, n, ws.pivots(), ws.blockOffsets(), ws.blockUniform(), ws.activeNbParts());
    ReduceBlockCounts<kMaxParts, 256><<<candidate, 256, 0, st>>>(ws.blockOffsets(), ws.blockUniform(),
                                                                 ws.counters() + 1, ws.uniformParts(), blocks,
                                                                 ws.activeNbParts());
    DetectSingleUniformBucket<<<1, 1, 0, st>>>(ws.counters() + 1, ws.uniformParts(), ws.activeNbParts(),
                                               ws.skipScatterFlag());
    BuildPrefixDynamic<int, kMaxParts><<<1, std::min(candidate, DefaultNbThreadsPerBlock), 0, st>>>(
        ws.counters() + 1, ws.activeNbParts());
    BuildPersistentBlockOffsets<kMaxParts><<<candidate, 1, 0, st>>>(ws.blockOffsets(), ws.counters(), blocks,
                                                                   ws.activeNbParts());
    MoveElements_Persistent<Elem, kMaxParts><<<blocks, DefaultNbThreadsPerBlock, 0, st>>>(
        data, n, ws.pivots(), ws.blockOffsets(), ws.valuesBuffer(), ws.activeNbParts(), ws.skipScatterFlag());
    int parts = 0, skipped = 0;
    cudaMemcpyAsync(&parts, ws.activeNbParts(), sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&skipped, ws.skipScatterFlag(), sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 2;
    if (skipped) {
        cudaMemcpyAsync(d_parts, data, size_t(n) * sizeof(Elem), cudaMemcpyDeviceToDevice, st);
        const int one[2] = {0, n};
        cudaMemcpyAsync(d_counters, one, sizeof(one), cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(d_uniform, 0xff, sizeof(int), st);
        parts = 1;
    } else {
        cudaMemcpyAsync(d_parts, ws.valuesBuffer(), size_t(n) * sizeof(Elem), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(d_counters, ws.counters(), (parts + 1) * sizeof(int), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(d_uniform, ws.uniformParts(), parts * sizeof(int), cudaMemcpyDeviceToDevice, st);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return 2;
    *nb_parts_out = parts;
    *skipped_out = skipped;
    return launch_status();
}

}  // extern "C"
