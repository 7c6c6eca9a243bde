// The transposed network for tiles of several warps: every comparator layer
// of an array held by a whole CTA (or one CTA's slice of a cluster's array)
// runs as a compare-exchange between two registers of one thread.
//
// The network is the reflection bitonic network of cusort_v6.hpp:90-142 (see
// network.cuh), with the keep-own rule of cusort.hpp:460-472: each
// comparator compares the same two elements as the reference's and puts the
// minimum at the lower logical index, so the output, tie order of records
// included, is the reference's.
//
// Layouts.  The slice of W = K * T elements (K = 2^LK per thread, T = 2^LT
// threads) has index bits [0, LK + LT).  In window layout A (0 <= A <= LT)
// register q of thread t holds the element of index
//     ((t >> A) << (A + LK)) | (q << A) | (t & (2^A - 1)),
// i.e. register bits are index bits A .. A+LK-1 and thread bits the others;
// A = 0 is the natural (blocked) layout of load_tile / store_tile.  Stage ST
// (span 2^ST) runs in registers when ST < LK.  Otherwise its layers run in a
// chain of windows: A1 = ST-LK+1 holds bits ST-LK+1 .. ST and is MIRRORED
// (registers whose index bit ST is set hold the element with index bits
// 0 .. ST-1 complemented), so the reflection pairs register q with q + K/2
// and the merges inside the mirrored half put the minimum in the upper
// register; then windows A1-LK, A1-2LK, ... (plain), the last one the
// natural layout, each running the merges on its register bits.  Between two
// windows the registers go through a per-slice shared region that stores the
// element of index i at xp_addr(i) = i + (i >> LK) (so a mirrored register
// lands at its logical place): one store and one load per element, no ALU
// work beyond a per-thread base per layout (register offsets are
// compile-time).  A stage of span 2^ST costs ceil((ST+1)/LK) such moves
// where the blocked network of network.cuh costs one shared-memory layer
// (store, load and a one-sided pick per element) per warp or lane bit.
//
// Bank conflicts.  With that padding every index bit b adds 2^b + 2^(b-LK)
// (b >= LK) to the address.  For 16-byte elements and LK = 4, and for 8-byte
// elements and LK = 4 or 5, the lane bits of a quarter-warp (half-warp) take
// weights of distinct 2-adic valuation modulo 8 (16) units in every layout,
// so each access instruction moves the minimum number of wavefronts.  (For
// 4-byte elements and LK = 4 the layouts A >= 5 have one two-way conflict.)
//
// Cluster stages (index bits above one CTA's slice) keep network.cuh's
// distributed-shared-memory layers (publish, cluster barrier, read the
// partner CTA's element, pick), run in window layout LT: there a warp's lanes
// read 32 consecutive elements of the partner's slice (in the blocked layout
// they were 2^LK + 1 elements apart, each read pulling a whole sector), and
// the registers hold the slice's top LK bits, so the first LK local merges
// need no layout change; the remaining merges run as a window chain.
//
// Keys alone (kKeysOnly) sort each thread's registers with Batcher's odd-even
// merge sort instead of stages 0 .. LK-1 (xpose.cuh); records keep the
// reference's comparators throughout.
#pragma once
#include <cooperative_groups.h>

#include "xpose.cuh"

namespace b200s {

// Per-thread base address of window A (plain, or mirrored: low thread bits
// complemented) and the compile-time offset of register q.
template <int LK, int A, bool MIR>
__device__ __forceinline__ int xc_base(int t) {
    constexpr int LOW = (1 << A) - 1;
    const int lo = MIR ? ((t & LOW) ^ LOW) : (t & LOW);
    return xp_addr<LK>(((t >> A) << (A + LK)) | lo);
}
template <int LK, int A, bool MIR>
__host__ __device__ constexpr int xc_off(int q) {
    constexpr int H = (1 << LK) >> 1;
    return xp_addr<LK>((MIR && (q & H) ? (q ^ (H - 1)) : q) << A);
}

template <class E, int LK, int A, bool MIR>
__device__ __forceinline__ void xc_put(const typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm) {
    constexpr int H = (1 << LK) >> 1;
    const int bp = xc_base<LK, A, false>(t);
    const int bm = MIR ? xc_base<LK, A, true>(t) : bp;
    sfor<0, (1 << LK)>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        sh_st(&sm[((MIR && (q & H)) ? bm : bp) + xc_off<LK, A, MIR>(q)], v[q]);
    });
}
template <class E, int LK, int A, bool MIR>
__device__ __forceinline__ void xc_get(typename E::Reg (&v)[1 << LK], const int t, const typename E::Reg* sm) {
    constexpr int H = (1 << LK) >> 1;
    const int bp = xc_base<LK, A, false>(t);
    const int bm = MIR ? xc_base<LK, A, true>(t) : bp;
    sfor<0, (1 << LK)>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        v[q] = sh_ld(&sm[((MIR && (q & H)) ? bm : bp) + xc_off<LK, A, MIR>(q)]);
    });
}

// Layout change through the single shared region: the first barrier lets
// every thread finish reading the region's previous contents.
template <class E, int LK, int AF, bool MF, int AT, bool MT, class Bar>
__device__ __forceinline__ void xc_move(typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm,
                                        const Bar& bar) {
    bar();
    xc_put<E, LK, AF, MF>(v, t, sm);
    bar();
    xc_get<E, LK, AT, MT>(v, t, sm);
}

// Plain merges on register bits R .. 0 of the current layout.
template <class E, int LK, int R>
__device__ __forceinline__ void xc_reg_merges(typename E::Reg (&v)[1 << LK]) {
    sfor<0, R + 1>([&](auto rc) {
        constexpr int r = R - decltype(rc)::value;
        sfor<0, (1 << LK)>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (!(q & (1 << r))) xcex<E, q>(v[q], v[q | (1 << r)]);
        });
    });
}

// From window ACUR (mirrored or not), the merges on index bits HI .. 0
// (HI = ACUR - 1 or below), ending in the natural layout.
template <class E, int LK, int ACUR, bool MCUR, int HI, class Bar>
__device__ __forceinline__ void xc_chain(typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm,
                                         const Bar& bar) {
    if constexpr (HI < 0) {
        if constexpr (ACUR != 0 || MCUR) xc_move<E, LK, ACUR, MCUR, 0, false>(v, t, sm, bar);
    } else {
        constexpr int AN = HI - LK + 1 > 0 ? HI - LK + 1 : 0;
        if constexpr (AN != ACUR || MCUR) xc_move<E, LK, ACUR, MCUR, AN, false>(v, t, sm, bar);
        xc_reg_merges<E, LK, HI - AN>(v);
        if constexpr (AN > 0) xc_chain<E, LK, AN, false, AN - 1>(v, t, sm, bar);
    }
}

// Stage ST of the slice's network (ST < LK + LT), natural layout in and out.
template <class E, int LK, int ST, class Bar>
__device__ __forceinline__ void xc_stage(typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm,
                                         const Bar& bar) {
    constexpr int K = 1 << LK, H = K >> 1;
    if constexpr (ST < LK) {
        // reflection and merges inside each thread's registers
        constexpr int M = (2 << ST) - 1;
        sfor<0, K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (q < (q ^ M)) xcex<E, q>(v[q], v[q ^ M]);
        });
        if constexpr (ST > 0) xc_reg_merges<E, LK, ST - 1>(v);
    } else {
        constexpr int A1 = ST - LK + 1;
        xc_move<E, LK, 0, false, A1, true>(v, t, sm, bar);
        // reflection: register q with its mirror partner q + K/2
        sfor<0, H>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            xcex<E, q>(v[q], v[q + H]);
        });
        // merges on index bits ST-1 .. A1 = register bits LK-2 .. 0; in the
        // mirrored half the lower logical index is the upper register
        sfor<0, LK - 1>([&](auto rc) {
            constexpr int r = LK - 2 - decltype(rc)::value;
            sfor<0, K>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                if constexpr (!(q & (1 << r))) {
                    if constexpr (q & H) xcex<E, q>(v[q | (1 << r)], v[q]);
                    else xcex<E, q>(v[q], v[q | (1 << r)]);
                }
            });
        });
        xc_chain<E, LK, A1, true, A1 - 1>(v, t, sm, bar);
    }
}

// The whole network of a slice of 2^LOGW elements (LOGW <= LK + LT).
template <class E, int LK, int LOGW, class Bar>
__device__ __forceinline__ void xc_network(typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm,
                                           const Bar& bar) {
    if constexpr (keys_only<E>::value) {
        xp_reg_sort_oem<E, LK>(v);  // keys alone: stages 0 .. LK-1 with fewer comparators
        sfor<LK, LOGW>([&](auto sc) { xc_stage<E, LK, decltype(sc)::value>(v, t, sm, bar); });
    } else {
        sfor<0, LOGW>([&](auto sc) { xc_stage<E, LK, decltype(sc)::value>(v, t, sm, bar); });
    }
}

// Shared-memory elements of a slice of 2^LOGW elements in this layout.
template <int LK, int LOGW>
constexpr int xc_smem_elems() {
    return xp_addr<LK>((1 << LOGW) - 1) + 1;
}

// Cross-CTA layer of a cluster stage, in window layout LT (register q of
// thread t holds local index (q << LT) | t, so the lanes of a warp read 32
// consecutive elements of the partner's slice): the partner of (rank, local
// index i) is (rank ^ cm, reflect ? i ^ (W - 1) : i).  The slice is
// published at its logical addresses, then read back from the partner CTA.
template <class E, int LK, int LT, bool REFLECT>
__device__ __forceinline__ void xc_cluster_layer(typename E::Reg (&v)[1 << LK], const int t, const int rank,
                                                 const int cm, const bool upper, typename E::Reg* sm) {
    using R = typename E::Reg;
    constexpr int K = 1 << LK, T = 1 << LT;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    xc_put<E, LK, LT, false>(v, t, sm);
    cluster.sync();
    const R* remote = cluster.map_shared_rank(sm, rank ^ cm);
    const int pb = xp_addr<LK>(REFLECT ? T - 1 - t : t);
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const R b = dsm_ld(&remote[pb + xp_addr<LK>((REFLECT ? K - 1 - q : q) << LT)]);
        v[q] = E::pick(v[q], b, upper);
    });
    cluster.sync();
}

// The network of an array held by a cluster of 2^LC CTAs of 2^LT threads
// (slice of 2^(LK+LT) elements per CTA): the local stages, then per cluster
// stage its cross-CTA layers in window layout LT, the merges on the slice's
// top LK bits in the same registers, and the rest as a window chain.
template <class E, int LK, int LT, int LC>
__device__ __forceinline__ void xc_cluster_network(typename E::Reg (&v)[1 << LK], const int t, const int rank,
                                                   typename E::Reg* sm) {
    constexpr int LOCAL = LK + LT;
    const CtaBarrier bar{};
    xc_network<E, LK, LOCAL>(v, t, sm, bar);
#pragma unroll 1
    for (int st = LOCAL; st < LOCAL + LC; ++st) {
        xc_move<E, LK, 0, false, LT, false>(v, t, sm, bar);
        __syncthreads();  // every thread has read the region before it is published again
        xc_cluster_layer<E, LK, LT, true>(v, t, rank, (2 << (st - LOCAL)) - 1, (rank >> (st - LOCAL)) & 1, sm);
#pragma unroll 1
        for (int j = st - 1; j >= LOCAL; --j)
            xc_cluster_layer<E, LK, LT, false>(v, t, rank, 1 << (j - LOCAL), (rank >> (j - LOCAL)) & 1, sm);
        // merges on local bits LOCAL-1 .. LT: the registers of window LT
        xc_reg_merges<E, LK, LK - 1>(v);
        xc_chain<E, LK, LT, false, LT - 1>(v, t, sm, bar);
    }
}

// One array per CTA of S::TPA threads (S::LW > 0), the grid striding over the
// batch; arguments and the sorted check as k_sort_packed's.
template <class E, class S, int MINB = 1>
__global__ void __launch_bounds__(S::TPA, MINB) k_sort_packed_xc(const typename E::Mem* in, typename E::Mem* out,
                                                                int n, long long arrays, unsigned opts) {
    using R = typename E::Reg;
    static_assert(S::LW > 0, "the transposed network of one warp is xpose.cuh's");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    const int t = int(threadIdx.x);
    // programmatic dependent launch (see k_sort_packed)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    for (long long a = blockIdx.x; a < arrays; a += gridDim.x) {
        const long long off = a * (long long)n;
        R v[S::K];
        load_tile<E, S::K>(v, in + off, t * S::K, n);
        const bool skip = (opts & kOptSortedCheck) && team_in_order<E, S>(v, t, sm);
        if (!skip) xc_network<E, S::LK, S::LOGW>(v, t, sm, CtaBarrier{});
        if (!skip || in != out) store_tile<E, S::K>(v, out + off, t * S::K, n);
        __syncthreads();  // the next array's first layout change reuses the region
    }
}

// k_sort_idlist with the transposed network (one array per CTA): the arrays
// ids[0 .. count) of a CSR batch, count and list position read on the device
// when d_count is set, CTAs pulling arrays from the queue at d_head when set.
template <class E, class S, int MINB = 1>
__global__ void __launch_bounds__(S::TPA, MINB)
    k_sort_idlist_xc(const typename E::Mem* in, typename E::Mem* out, const int* __restrict__ off,
                     const int* __restrict__ ids, int count, const int* d_count, const int* d_base, int* d_head) {
    using R = typename E::Reg;
    static_assert(S::LW > 0, "one array per CTA");
    __shared__ int s_next;
    if (d_count) {
        count = *d_count;
        ids += *d_base;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    const int t = int(threadIdx.x);
    long long g = blockIdx.x;
    for (;;) {
        if (d_head) {
            if (t == 0) s_next = atomicAdd(d_head, 1);
            __syncthreads();
            g = s_next;
            __syncthreads();
        }
        if (g >= count) break;  // uniform across the CTA
        const int a = ids[g];
        const long long start = off[a];
        const int na = off[a + 1] - off[a];
        R v[S::K];
        load_tile<E, S::K>(v, in + start, t * S::K, na);
        xc_network<E, S::LK, S::LOGW>(v, t, sm, CtaBarrier{});
        store_tile<E, S::K>(v, out + start, t * S::K, na);
        __syncthreads();
        if (!d_head) g += gridDim.x;
    }
}

// One cluster of 2^LC CTAs per array, clusters striding over the batch, with
// the transposed network; the arguments are k_sort_cluster's (packed batch
// when ids == nullptr, else the CSR arrays ids[0 .. count)).  Every warp runs
// the whole network (a window layout mixes padding with elements, so warps of
// padding cannot skip layers as in network.cuh's compact form).
template <class E, int LK, int LT, int LC, int MINB = 1>
__global__ void __launch_bounds__(1 << LT, MINB)
    k_sort_cluster_xc(const typename E::Mem* in, typename E::Mem* out, int n, long long arrays, const int* off,
                      const int* ids, const int* d_count) {
    using R = typename E::Reg;
    namespace cg = cooperative_groups;
    constexpr int K = 1 << LK, W = 1 << (LK + LT);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
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
        const int base = rank * W + t * K;
        R v[K];
        load_tile<E, K>(v, in + start, base, na);
        xc_cluster_network<E, LK, LT, LC>(v, t, rank, sm);
        store_tile<E, K>(v, out + start, base, na);
    }
}

}  // namespace b200s
