// Launch form 3 of multi-warp and cluster tiles: the transposed network of
// cta_xpose.cuh attached to the registered entries of the same shapes.  Only
// the xc_*.cu translation units include this header.
#pragma once
#include <type_traits>

#include "cta_xpose.cuh"
#include "instantiate.cuh"

namespace b200s {

// Launch form 3 of the multi-warp tile Shape<LK, 5, LW> (one array per CTA):
// the transposed network, attached to that tile's registry entry.
template <class E, int LK, int LW, int MINB = 1>
struct PackedXc {
    using S = Shape<LK, 5, LW>;
    static_assert(LW > 0, "multi-warp tiles");
    static constexpr int CTA = S::TPA;
    static constexpr size_t SMEM = size_t(xc_smem_elems<LK, S::LOGW>()) * sizeof(typename E::Reg);
    static cudaError_t launch(const void* in, void* out, int n, long long arrays, long long,
                              cudaStream_t st, unsigned opts) {
        static std::atomic<unsigned long long> done{0};
        auto fn = k_sort_packed_xc<E, S, MINB>;
        cudaError_t e = opt_in_smem<SMEM>(reinterpret_cast<const void*>(fn), done);
        if (e != cudaSuccess) return e;
        const long long grid = arrays < 0x7fffffffLL ? arrays : 0x7fffffffLL;
        return launch_pdl(fn, unsigned(grid), CTA, SMEM, st, static_cast<const typename E::Mem*>(in),
                          static_cast<typename E::Mem*>(out), n, arrays, opts);
    }
    static cudaError_t launch_list(const void* in, void* out, const int* off, const int* ids, int count,
                                   cudaStream_t st) {
        static std::atomic<unsigned long long> done{0};
        auto fn = k_sort_idlist_xc<E, S, MINB>;
        cudaError_t e = opt_in_smem<SMEM>(reinterpret_cast<const void*>(fn), done);
        if (e != cudaSuccess) return e;
        fn<<<dim3(unsigned(count > 0 ? count : 1)), dim3(CTA), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), off, ids, count, nullptr,
            nullptr, nullptr);
        return cudaGetLastError();
    }
    static cudaError_t launch_list_dev(const void* in, void* out, const int* off, const int* ids, const int* d_count,
                                       const int* d_base, int* d_head, int max_count, cudaStream_t st) {
        static std::atomic<unsigned long long> done{0};
        static std::atomic<int> resident[64];
        auto fn = k_sort_idlist_xc<E, S, MINB>;
        cudaError_t e = opt_in_smem<SMEM>(reinterpret_cast<const void*>(fn), done);
        if (e != cudaSuccess) return e;
        int cap = 0;
        if ((e = resident_ctas(reinterpret_cast<const void*>(fn), CTA, SMEM, resident, &cap)) != cudaSuccess)
            return e;
        const int grid = max_count < cap ? (max_count > 0 ? max_count : 1) : cap;
        fn<<<dim3(unsigned(grid)), dim3(CTA), SMEM, st>>>(static_cast<const typename E::Mem*>(in),
                                                          static_cast<typename E::Mem*>(out), off, ids, 0, d_count,
                                                          d_base, d_head);
        return cudaGetLastError();
    }
    // Attach to the registered single-CTA entry of this shape and type.
    static void attach_to(std::vector<KernelEntry>& o, int dtype) {
        for (KernelEntry& k : o)
            if (k.dtype == dtype && k.stable == (E::kStable ? 1 : 0) && k.lk == LK && k.lg == 5 && k.lw == LW &&
                k.lc < 0) {
                k.launch_xc = &launch;
                k.launch_list_xc = &launch_list;
                k.launch_list_dev_xc = &launch_list_dev;
                k.smem_xc = SMEM;
            }
    }
};

// The cluster kernel of the transposed network, as ClusterTile's KERNEL.
struct ClusterXcKernel {
    template <class E, int LK, int LT, int LC, int MINB>
    static constexpr auto fn() {
        return k_sort_cluster_xc<E, LK, LT, LC, MINB>;
    }
};

// Launch form 3 of the cluster tile ClusterTile<E, LK, LG, LW, LC, SB>.
template <class E, int LK, int LG, int LW, int LC, bool SB, int MINB = 1>
struct ClusterXc {
    using Tile = ClusterTile<E, LK, LG, LW, LC, SB, MINB, ClusterXcKernel,
                             size_t(xc_smem_elems<LK, LK + LG + LW>())>;
    // Attach to the registered cluster entry of the same shape, CTAs per
    // array and dtype (whose element type may be another of the same
    // records, e.g. a compact form).
    static void attach_to(std::vector<KernelEntry>& o, int dtype) {
        for (KernelEntry& k : o)
            if (k.dtype == dtype && k.stable == (E::kStable ? 1 : 0) && k.lk == LK && k.lg == LG && k.lw == LW &&
                k.lc == LC) {
                k.launch_xc = &Tile::launch;
                k.launch_list_xc = &Tile::launch_list;
                k.launch_cluster_list_xc = &Tile::launch_cluster_list;
                k.smem_xc = Tile::SMEM;
                // a cluster of one CTA is a single-CTA tile: a ragged length
                // class can run it as a launch of its own with the queue
                if constexpr (LC == 0 && LG == 5 && LW > 0) k.launch_list_dev_xc = &PackedXc<E, LK, LW, MINB>::launch_list_dev;
            }
    }
};

}  // namespace b200s
