// Kernel instantiation helpers shared by the per-type translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

#include "network.cuh"
#include "registry.h"

namespace b200s {

// Ragged-list kernel: CTA-group g sorts array ids[g] whose elements start at
// start[id] and number len[id].  Used by the per-bucket launches of a plan.
template <class E, class S, int CTA>
__global__ void __launch_bounds__(CTA) k_sort_list(const typename E::Mem* in, typename E::Mem* out,
                                                   const long long* start, const int* len,
                                                   const int* ids, long long count) {
    using R = typename E::Reg;
    constexpr int APC = CTA / S::TPA;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* cur = reinterpret_cast<R*>(smem_raw);
    R* nxt = cur + S::W;
    const int slot = int(threadIdx.x) / S::TPA;
    const int t = int(threadIdx.x) % S::TPA;
    for (long long first = (long long)blockIdx.x * APC; first < count;
         first += (long long)gridDim.x * APC) {
        const long long g = first + slot;
        int na = 0;
        long long off = 0;
        if (g < count) {
            const int id = ids[g];
            na = len[id];
            off = start[id];
        }
        R v[S::K];
        load_tile<E, S::K>(v, in + off, t * S::K, na);
        network<E, S>(v, t, cur, nxt);
        store_tile<E, S::K>(v, out + off, t * S::K, na);
    }
}

template <class E, int LK, int LG, int LW>
struct Packed {
    using S = Shape<LK, LG, LW>;
    static constexpr int CTA = LW > 0 ? S::TPA : (S::TPA >= 128 ? S::TPA : 128);
    static constexpr size_t SMEM = LW > 0 ? 2 * size_t(S::W) * sizeof(typename E::Reg) : 0;

    static cudaError_t prepare(const void* fn) {
        if (SMEM <= 48 * 1024) return cudaSuccess;
        // The opt-in above 48 KB is per device; remember which devices have it.
        static std::atomic<unsigned long long> done{0};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const unsigned long long bit = 1ull << (dev & 63);
        if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM));
        if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
        return e;
    }
    static cudaError_t launch(const void* in, void* out, int n, long long arrays, long long grid,
                              cudaStream_t st) {
        auto fn = k_sort_packed<E, S, CTA>;
        cudaError_t e = prepare(reinterpret_cast<const void*>(fn));
        if (e != cudaSuccess) return e;
        fn<<<dim3(unsigned(grid)), dim3(CTA), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), n, arrays);
        return cudaGetLastError();
    }
    static cudaError_t launch_list(const void* in, void* out, const long long* start, const int* len,
                                   const int* ids, long long count, long long grid,
                                   cudaStream_t st) {
        auto fn = k_sort_list<E, S, CTA>;
        cudaError_t e = prepare(reinterpret_cast<const void*>(fn));
        if (e != cudaSuccess) return e;
        fn<<<dim3(unsigned(grid)), dim3(CTA), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), start, len,
            ids, count);
        return cudaGetLastError();
    }
    // Persistent launch: as many CTAs as fit at once (cached per device), never
    // more than the batch needs.
    static cudaError_t launch_pf(const void* in, void* out, int n, long long arrays, long long grid,
                                 cudaStream_t st) {
        auto fn = k_sort_packed_pf<E, S, CTA>;
        cudaError_t e = prepare(reinterpret_cast<const void*>(fn));
        if (e != cudaSuccess) return e;
        static std::atomic<int> resident[64];
        int dev = 0;
        e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        int cap = resident[dev & 63].load(std::memory_order_relaxed);
        if (cap == 0) {
            int per_sm = 0, sms = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, CTA, SMEM);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            cap = per_sm * sms;
            if (cap <= 0) return cudaErrorInvalidConfiguration;
            resident[dev & 63].store(cap, std::memory_order_relaxed);
        }
        const long long g = grid < cap ? grid : cap;
        fn<<<dim3(unsigned(g)), dim3(CTA), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), n, arrays);
        return cudaGetLastError();
    }
    static cudaError_t attrs(cudaFuncAttributes* a) {
        return cudaFuncGetAttributes(a, reinterpret_cast<const void*>(k_sort_packed<E, S, CTA>));
    }
    static KernelEntry entry(int dtype) {
        return KernelEntry{dtype,   E::kStable ? 1 : 0, LK,     LG,         LW,
                           CTA,     S::LOGW,            SMEM,   CTA / S::TPA, &launch,
                           &attrs,  &launch_list,       &launch_pf};
    }
};

}  // namespace b200s
