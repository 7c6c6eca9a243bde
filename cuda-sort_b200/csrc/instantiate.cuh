// Kernel instantiation helpers shared by the per-type translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <type_traits>

#include "cluster.cuh"
#include "network.cuh"
#include "ragged.cuh"
#include "registry.h"

namespace b200s {

// Launch with programmatic stream serialization allowed (the kernel starts
// with griddepcontrol.wait, so it still sees all of the previous kernel's
// writes).
template <class... P, class... A>
cudaError_t launch_pdl(void (*fn)(P...), unsigned grid, int cta, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(unsigned(cta));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, fn, args...);
}

// SB: single-buffered shared-memory layers (multi-warp tiles only).
template <class E, int LK, int LG, int LW, bool SB = false>
struct Packed {
    using S = Shape<LK, LG, LW>;
    static constexpr int CTA = LW > 0 ? S::TPA : (S::TPA >= 128 ? S::TPA : 128);
    static constexpr size_t SMEM = LW > 0 ? (SB ? 1 : 2) * size_t(S::W) * sizeof(typename E::Reg) : 0;

    // The opt-in above 48 KB is per kernel and per device; WHICH keeps one
    // record per kernel of this tile (0 packed, 1 list, 2 persistent).
    template <int WHICH>
    static cudaError_t prepare(const void* fn) {
        // the default limit covers static + dynamic shared memory: opt in
        // with a margin for the kernels' own static variables
        if (SMEM + 1024 <= 48 * 1024) return cudaSuccess;
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
    // Programmatic dependent launch: the grid may be scheduled while the
    // stream's previous kernel drains (the kernel waits for it first).
    static cudaError_t launch(const void* in, void* out, int n, long long arrays, long long grid,
                              cudaStream_t st, unsigned opts) {
        auto fn = k_sort_packed<E, S, CTA, SB>;
        cudaError_t e = prepare<0>(reinterpret_cast<const void*>(fn));
        if (e != cudaSuccess) return e;
        return launch_pdl(fn, unsigned(grid), CTA, SMEM, st, static_cast<const typename E::Mem*>(in),
                          static_cast<typename E::Mem*>(out), n, arrays, opts);
    }
    static cudaError_t launch_list(const void* in, void* out, const int* off, const int* ids, int count,
                                   cudaStream_t st) {
        auto fn = k_sort_idlist<E, S, CTA, SB>;  // the same buffering as SMEM
        cudaError_t e = prepare<1>(reinterpret_cast<const void*>(fn));
        if (e != cudaSuccess) return e;
        const int grid = (count + CTA / S::TPA - 1) / (CTA / S::TPA);
        fn<<<dim3(unsigned(grid)), dim3(CTA), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), off, ids, count, nullptr,
            nullptr, nullptr);
        return cudaGetLastError();
    }
    // Over a dedicated bucket of a ragged plan: count and list position read
    // on the device; the grid is the resident capacity (cached per device),
    // at most what max_count arrays need, pulling arrays from the queue at
    // d_head (zero before the launch).
    static cudaError_t launch_list_dev(const void* in, void* out, const int* off, const int* ids, const int* d_count,
                                       const int* d_base, int* d_head, int max_count, cudaStream_t st) {
        auto fn = k_sort_idlist<E, S, CTA, SB>;
        cudaError_t e = prepare<1>(reinterpret_cast<const void*>(fn));
        if (e != cudaSuccess) return e;
        static std::atomic<int> resident[64];
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        int cap = resident[dev & 63].load(std::memory_order_relaxed);
        if (cap == 0) {
            int per_sm = 0, sms = 0;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, CTA, SMEM)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            cap = per_sm * sms;
            if (cap <= 0) return cudaErrorInvalidConfiguration;
            resident[dev & 63].store(cap, std::memory_order_relaxed);
        }
        const int need = (max_count + CTA / S::TPA - 1) / (CTA / S::TPA);
        const int grid = need < cap ? (need > 0 ? need : 1) : cap;
        fn<<<dim3(unsigned(grid)), dim3(CTA), SMEM, st>>>(static_cast<const typename E::Mem*>(in),
                                                          static_cast<typename E::Mem*>(out), off, ids, 0, d_count,
                                                          d_base, d_head);
        return cudaGetLastError();
    }
    // Persistent launch: as many CTAs as fit at once (cached per device), never
    // more than the batch needs.
    static cudaError_t launch_pf(const void* in, void* out, int n, long long arrays, long long grid,
                                 cudaStream_t st, unsigned opts) {
        auto fn = k_sort_packed_pf<E, S, CTA, SB>;
        cudaError_t e = prepare<2>(reinterpret_cast<const void*>(fn));
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
        return launch_pdl(fn, unsigned(g), CTA, SMEM, st, static_cast<const typename E::Mem*>(in),
                          static_cast<typename E::Mem*>(out), n, arrays, opts);
    }
    static cudaError_t attrs(cudaFuncAttributes* a) {
        return cudaFuncGetAttributes(a, reinterpret_cast<const void*>(k_sort_packed<E, S, CTA, SB>));
    }
    static KernelEntry entry(int dtype) {
        return KernelEntry{dtype,   E::kStable ? 1 : 0, LK,     LG,         LW,
                           CTA,     S::LOGW,            SMEM,   CTA / S::TPA, &launch,
                           &attrs,  &launch_list,       &launch_pf, -1,   nullptr, &launch_list_dev};
    }
};

// Opt in to SMEM bytes of dynamic shared memory for kernel fn (once per
// device), with a margin for the kernel's own static variables.
template <size_t SMEM>
cudaError_t opt_in_smem(const void* fn, std::atomic<unsigned long long>& done) {
    if (SMEM + 1024 <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM));
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// CTAs of kernel fn resident at once on the current device (cached per device
// in cache[]).
inline cudaError_t resident_ctas(const void* fn, int cta, size_t smem, std::atomic<int>* cache, int* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int cap = cache[dev & 63].load(std::memory_order_relaxed);
    if (cap == 0) {
        int per_sm = 0, sms = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, cta, smem)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        cap = per_sm * sms;
        if (cap <= 0) return cudaErrorInvalidConfiguration;
        cache[dev & 63].store(cap, std::memory_order_relaxed);
    }
    *out = cap;
    return cudaSuccess;
}

// A cluster of 2^LC CTAs per array (SB: single-buffered shared memory).
// KERNEL: the kernel template with k_sort_cluster's parameters and
// arguments; SMEM_ELEMS its shared-memory elements per CTA (0: SB ? W : 2W).
// Launch form 3 (instantiate_xc.cuh) reuses this with the transposed network.
template <class E, int LK, int LG, int LW, int LC, bool SB, int MINB = 1, class KERNEL = void,
          size_t SMEM_ELEMS = 0>
struct ClusterTile {
    using S = Shape<LK, LG, LW>;
    static constexpr int CTA = S::TPA;
    static constexpr int C = 1 << LC;
    static constexpr size_t SMEM = SMEM_ELEMS ? SMEM_ELEMS * sizeof(typename E::Reg)
                                              : (SB ? 1 : 2) * size_t(S::W) * sizeof(typename E::Reg);
    static constexpr auto kernel() {
        if constexpr (std::is_void_v<KERNEL>) return k_sort_cluster<E, S, LC, SB, MINB>;
        else return KERNEL::template fn<E, LK, LG + LW, LC, MINB>();
    }

    static cudaLaunchConfig_t config(long long clusters, cudaStream_t st, cudaLaunchAttribute* attr) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(clusters * C), 1, 1);
        cfg.blockDim = dim3(CTA, 1, 1);
        cfg.dynamicSmemBytes = SMEM;
        cfg.stream = st;
        attr->id = cudaLaunchAttributeClusterDimension;
        attr->val.clusterDim.x = C;
        attr->val.clusterDim.y = 1;
        attr->val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cfg;
    }
    // Clusters resident at once on this device (cached per device).
    static cudaError_t resident(int* out) {
        static std::atomic<int> cache[64];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        int v = cache[dev & 63].load(std::memory_order_relaxed);
        if (v == 0) {
            auto fn = kernel();
            e = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(SMEM));
            if (e != cudaSuccess) return e;
            cudaLaunchAttribute attr;
            cudaLaunchConfig_t cfg = config(1, nullptr, &attr);
            e = cudaOccupancyMaxActiveClusters(&v, fn, &cfg);
            if (e != cudaSuccess) return e;
            if (v <= 0) return cudaErrorInvalidConfiguration;
            cache[dev & 63].store(v, std::memory_order_relaxed);
        }
        *out = v;
        return cudaSuccess;
    }
    static cudaError_t run(const void* in, void* out, int n, long long arrays, const int* off, const int* ids,
                           const int* d_count, long long clusters, cudaStream_t st) {
        int cap = 0;
        cudaError_t e = resident(&cap);
        if (e != cudaSuccess) return e;
        clusters = clusters < cap ? clusters : cap;
        if (clusters < 1) clusters = 1;
        cudaLaunchAttribute attr;
        cudaLaunchConfig_t cfg = config(clusters, st, &attr);
        return cudaLaunchKernelEx(&cfg, kernel(), static_cast<const typename E::Mem*>(in),
                                  static_cast<typename E::Mem*>(out), n, arrays, off, ids, d_count);
    }
    static cudaError_t launch(const void* in, void* out, int n, long long arrays, long long, cudaStream_t st,
                              unsigned) {
        return run(in, out, n, arrays, nullptr, nullptr, nullptr, arrays, st);
    }
    static cudaError_t launch_list(const void* in, void* out, const int* off, const int* ids, int count,
                                   cudaStream_t st) {
        return run(in, out, 0, count, off, ids, nullptr, count, st);
    }
    static cudaError_t launch_cluster_list(const void* in, void* out, const int* off, const int* ids,
                                           const int* d_count, int max_count, cudaStream_t st) {
        return run(in, out, 0, max_count, off, ids, d_count, max_count, st);
    }
    static cudaError_t attrs(cudaFuncAttributes* a) {
        return cudaFuncGetAttributes(a, reinterpret_cast<const void*>(kernel()));
    }
    static KernelEntry entry(int dtype) {
        return KernelEntry{dtype, E::kStable ? 1 : 0, LK, LG, LW, CTA, S::LOGW + LC, SMEM, 1, &launch, &attrs,
                           &launch_list, &launch, LC, &launch_cluster_list, nullptr};
    }
};

// The persistent ragged kernel of element type E.
template <class E, int CTA, int NB, int LKA, int LKB, bool SB = false, int MINB = 1>
struct Ragged {
    static constexpr size_t SMEM = ragged_smem<E, CTA, NB, LKA, LKB, SB>();
    static cudaError_t launch(const void* in, void* out, const int* off, const int* ids, RaggedCtl* ctl,
                              unsigned family_mask, unsigned dedicated_mask, int grid, cudaStream_t st) {
        auto fn = k_sort_ragged<E, CTA, NB, LKA, LKB, SB, MINB>;
        if (SMEM > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM));
            if (e != cudaSuccess) return e;
        }
        fn<<<dim3(unsigned(grid)), dim3(CTA), SMEM, st>>>(static_cast<const typename E::Mem*>(in),
                                                          static_cast<typename E::Mem*>(out), off, ids, ctl,
                                                          family_mask, dedicated_mask);
        return cudaGetLastError();
    }
    static int resident_per_sm() {
        auto fn = k_sort_ragged<E, CTA, NB, LKA, LKB, SB, MINB>;
        if (SMEM > 48 * 1024 &&
            cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(SMEM)) != cudaSuccess)
            return 0;
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, CTA, SMEM) != cudaSuccess) return 0;
        return per_sm;
    }
    static RaggedEntry entry(int dtype) {
        return RaggedEntry{dtype, E::kStable ? 1 : 0, CTA, NB, LKA, LKB, SMEM, &launch, &resident_per_sm};
    }
};

}  // namespace b200s
