// Arrays larger than one CTA: a thread-block cluster of C = 2^LC CTAs sorts
// one array, exchanging through distributed shared memory.
//
// The working tile of W = 2^(LK+LG+LW+LC) elements is split into C slices of
// W/C consecutive elements, one per CTA of the cluster (index bits above
// LK+LG+LW select the CTA rank).  Comparator layers whose partner is in the
// same CTA run as in the single-CTA kernels (registers, shuffles, shared
// memory).  A layer whose partner is in another CTA publishes the tile into
// this CTA's shared memory, waits on the cluster barrier, reads the partner
// elements straight from the partner CTA's shared memory
// (cluster.map_shared_rank, i.e. ld.shared::cluster), and waits on the
// cluster barrier again before any buffer is reused.  No TMA is involved.
//
// The reference sorts an array larger than one block only as a single large
// array (SortMerge, cusort.hpp:2161-2300: chunk sorts plus log2(n/chunk)
// merge-path passes through global memory); here the whole network of such
// an array stays on chip.
#pragma once
#include <cooperative_groups.h>

#include "network.cuh"

namespace b200s {

namespace cg = cooperative_groups;

template <class E, class S, int LC, unsigned MASK, bool SB>
__device__ __forceinline__ void cluster_layer(typename E::Reg (&v)[S::K], const int t, const int rank,
                                              typename E::Reg*& cur, typename E::Reg*& nxt) {
    using R = typename E::Reg;
    constexpr int LOCAL = S::LOGW;
    constexpr int HB = hibit(MASK);
    if constexpr (HB < LOCAL) {
        if constexpr (SB) layer<E, S, MASK>(v, t, cur, nxt, CtaBarrierSingle{});
        else layer<E, S, MASK>(v, t, cur, nxt, CtaBarrier{});
    } else {
        constexpr unsigned RM = MASK & unsigned(S::K - 1);
        constexpr unsigned TM = (MASK >> S::LK) & unsigned(S::TPA - 1);
        constexpr unsigned CM = MASK >> LOCAL;
        cg::cluster_group cluster = cg::this_cluster();
        const bool upper = (rank >> (HB - LOCAL)) & 1;
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            sh_st(&cur[q * S::TPA + t], v[q]);
        });
        cluster.sync();
        const R* remote = cluster.map_shared_rank(cur, int(unsigned(rank) ^ CM));
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const R b = dsm_ld(&remote[(q ^ int(RM)) * S::TPA + (t ^ int(TM))]);
            v[q] = E::pick(v[q], b, upper);
        });
        cluster.sync();
    }
}

// Cross-CTA layer with a run-time CTA mask cm: the partner of (rank, t, q)
// is (rank ^ cm, t ^ TM, q ^ RM); a reflection flips every lower bit (RM, TM
// all ones), a merge only the CTA bit.
// Cluster barrier for warps that reach it from different code (no .aligned):
// arrive with release, wait with acquire semantics at cluster scope.
__device__ __forceinline__ void cluster_sync_unaligned() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// LIVE == false: the copy run by a warp that holds only padding; it
// publishes and meets both cluster barriers but reads nothing.  UA: warps of
// the cluster run different copies (unaligned barriers).
template <class E, class S, unsigned RM, unsigned TM, bool LIVE, bool UA>
__device__ __forceinline__ void cta_layer_rt(typename E::Reg (&v)[S::K], const int t, const int rank, const int cm,
                                             const bool upper, typename E::Reg* cur) {
    using R = typename E::Reg;
    cg::cluster_group cluster = cg::this_cluster();
    sfor<0, S::K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        sh_st(&cur[q * S::TPA + t], v[q]);
    });
    if constexpr (UA) cluster_sync_unaligned();
    else cluster.sync();
    if constexpr (LIVE) {
        const R* remote = cluster.map_shared_rank(cur, rank ^ cm);
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const R b = dsm_ld(&remote[(q ^ int(RM)) * S::TPA + (t ^ int(TM))]);
            v[q] = E::pick(v[q], b, upper);
        });
    }
    if constexpr (UA) cluster_sync_unaligned();
    else cluster.sync();
}

// The cluster network with the stages above one CTA as a run-time loop
// (one copy of their code), for elements whose unrolled network would not
// fit the instruction cache.  LIVE == false: the copy for a warp that holds
// only padding (see network_compact): it publishes and synchronises only,
// through the same barriers in the same order.
template <class E, class S, int LC, bool SB, bool LIVE, bool UA>
__device__ __forceinline__ void cluster_network_compact(typename E::Reg (&v)[S::K], const int t, const int rank,
                                                        typename E::Reg*& cur, typename E::Reg*& nxt) {
    constexpr int LOCAL = S::LOGW;
    // stages inside one CTA
    if constexpr (SB) network_compact<E, S, LIVE, UA>(v, t, cur, nxt, CtaBarrierSingle{});
    else network_compact<E, S, LIVE, UA>(v, t, cur, nxt, CtaBarrier{});
#pragma unroll 1
    for (int st = LOCAL; st < LOCAL + LC; ++st) {
        cta_layer_rt<E, S, unsigned(S::K - 1), unsigned(S::TPA - 1), LIVE, UA>(
            v, t, rank, (2 << (st - LOCAL)) - 1, (rank >> (st - LOCAL)) & 1, cur);
#pragma unroll 1
        for (int j = st - 1; j >= LOCAL; --j)
            cta_layer_rt<E, S, 0u, 0u, LIVE, UA>(v, t, rank, 1 << (j - LOCAL), (rank >> (j - LOCAL)) & 1, cur);
        // merges inside the CTA: warp and lane bits at run time, then registers
#pragma unroll 1
        for (int j = LOCAL - 1; j >= S::LK; --j) {
            if constexpr (SB) cross_layer_rt<E, S, 0u, LIVE, UA>(v, t, j, cur, nxt, CtaBarrierSingle{});
            else cross_layer_rt<E, S, 0u, LIVE, UA>(v, t, j, cur, nxt, CtaBarrier{});
        }
        if constexpr (LIVE) {
            sfor<0, S::LK>([&](auto jc) {
                constexpr int j = S::LK - 1 - decltype(jc)::value;
                layer<E, S, (1u << j)>(v, t, cur, nxt, CtaBarrier{});
            });
        }
    }
}

// n: the array's length.  The compact form gives warps of padding the copy
// that only publishes and synchronises, and runs arrays without such warps
// through the copy with aligned barriers; the unrolled form, kept for int32
// keys, runs every warp through the whole network.
template <class E, class S, int LC, bool SB>
__device__ __forceinline__ void cluster_network(typename E::Reg (&v)[S::K], const int t, const int rank,
                                                typename E::Reg*& cur, typename E::Reg*& nxt, const long long n) {
    if constexpr (use_compact<E, S>()) {
        constexpr long long kLastWarp = (long long)((1 << LC) - 1) * S::W;
        if (warp_live<S>(S::TPA - 1, n, kLastWarp)) cluster_network_compact<E, S, LC, SB, true, false>(v, t, rank, cur, nxt);
        else if (warp_live<S>(t, n, (long long)rank * S::W)) cluster_network_compact<E, S, LC, SB, true, true>(v, t, rank, cur, nxt);
        else cluster_network_compact<E, S, LC, SB, false, true>(v, t, rank, cur, nxt);
    } else {
        constexpr int LOGW = S::LOGW + LC;
        sfor<0, LOGW>([&](auto sc) {
            constexpr int ST = decltype(sc)::value;
            cluster_layer<E, S, LC, (2u << ST) - 1u, SB>(v, t, rank, cur, nxt);
            sfor<0, ST>([&](auto jc) {
                constexpr int j = ST - 1 - decltype(jc)::value;
                cluster_layer<E, S, LC, (1u << j), SB>(v, t, rank, cur, nxt);
            });
        });
    }
}

// One cluster per array, clusters striding over the batch.  Packed batches
// (ids == nullptr): array a at a*n, count = arrays.  Id lists: array ids[i]
// of a CSR batch, count read from *d_count (or `arrays` when d_count is null).
// MINB: CTAs per SM the register budget is sized for (2 with single-buffered
// shared memory lets two clusters' CTAs share an SM).
template <class E, class S, int LC, bool SB, int MINB = 1>
__global__ void __launch_bounds__(S::TPA, MINB) k_sort_cluster(const typename E::Mem* in, typename E::Mem* out,
                                                            int n, long long arrays, const int* off,
                                                            const int* ids, const int* d_count) {
    using R = typename E::Reg;
    static_assert(S::LW > 0 || S::LG == 5, "a cluster CTA holds whole warps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* cur = reinterpret_cast<R*>(smem_raw);
    R* nxt = SB ? cur : cur + S::W;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = int(cluster.block_rank());
    const int t = int(threadIdx.x);
    const long long cid = (long long)blockIdx.x >> LC;
    const long long clusters = (long long)gridDim.x >> LC;
    const long long count = ids ? (d_count ? (long long)*d_count : arrays) : arrays;
    for (long long i = cid; i < count; i += clusters) {
        long long start;
        int na;
        if (ids) {
            const int a = ids[i];
            start = off[a];
            na = off[a + 1] - off[a];
        } else {
            start = i * (long long)n;
            na = n;
        }
        const int base = rank * S::W + t * S::K;
        R v[S::K];
        load_tile<E, S::K>(v, in + start, base, na);
        cluster_network<E, S, LC, SB>(v, t, rank, cur, nxt, na);
        store_tile<E, S::K>(v, out + start, base, na);
    }
}

}  // namespace b200s
