// Ragged (CSR) batches in one persistent, length-bucketed launch.
//
// Array a occupies elements [off[a], off[a+1]) of the flat buffer.  The
// launch sequence of a plan is
//   1. reset the control block (counters, queue head),
//   2. k_bin_count   - histogram of arrays per working-length bucket,
//   3. k_bin_scatter - array ids grouped by bucket, largest bucket first,
//   4. k_sort_ragged - persistent CTAs pull tasks from a device queue (one
//                      atomicAdd per task; no waiting on other CTAs).  A task
//                      is one CTA's worth of arrays of one bucket: the CTA
//                      splits into teams of TPA threads, one array per team,
//                      each team running the bitonic network of its bucket's
//                      tile (multi-warp teams synchronise on a named barrier).
// Tasks are ordered largest working length first, so the longest tasks start
// early and the short ones fill the tail.  The bitonic network's cost depends
// only on the working length, so all teams of a task finish together.
//
// The reference's only ragged one-launch precedent is
// SortPartitionsAdaptive_outofplace (cusort.hpp:2309-2352), a grid-stride loop
// over CSR partitions with one block shape and shared memory sized for the
// largest partition; here every bucket has its own tile shape.
#pragma once
#include <cuda_runtime.h>

#include "network.cuh"

namespace b200s {

constexpr int kMaxBuckets = 16;
constexpr int kMaxOverflow = 4;
constexpr int kRaggedLmin = 3;  // smallest bucket: W = 8

struct RaggedCtl {
    int count[kMaxBuckets];    // arrays per bucket
    int cursor[kMaxBuckets];   // scatter cursors
    int base[kMaxBuckets];     // first position of each bucket's ids in the id list
    int dhead[kMaxBuckets];    // work queue heads of the dedicated bucket launches
    int head;                  // task queue head
    int too_long;              // arrays longer than every kernel (not sorted)
    int ocount[kMaxOverflow];  // arrays per cluster bucket
    int reserved[2];
};

// Binning parameters: nb buckets for the persistent kernel (W = 8 .. 8 <<
// (nb-1)); arrays with log2 W in [over_lo, over_lo + n_over) go to the
// cluster bucket log2 W - over_lo (ids at oids[bucket * stride]).
struct BinSpec {
    int nb;
    int over_lo;
    int n_over;
    int stride;
};

__device__ __forceinline__ int ceil_log2_dev(int n) { return n <= 1 ? 0 : 32 - __clz(n - 1); }

// Bucket of an array of length n >= 1: log2 of its working length, minus lmin.
__device__ __forceinline__ int bucket_of(int n, int lmin) {
    const int l = ceil_log2_dev(n);
    return (l > lmin ? l : lmin) - lmin;
}

// The binning kernels are defined in exactly one translation unit (plan.cu).
#ifdef B200S_DEFINE_BIN_KERNELS
__global__ void k_bin_count(const int* __restrict__ off, int arrays, RaggedCtl* ctl, BinSpec spec) {
    __shared__ int h[kMaxBuckets];
    __shared__ int over;
    if (threadIdx.x < kMaxBuckets) h[threadIdx.x] = 0;
    if (threadIdx.x == 0) over = 0;
    __syncthreads();
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < arrays; a += gridDim.x * blockDim.x) {
        const int n = off[a + 1] - off[a];
        if (n <= 0) continue;
        const int b = bucket_of(n, kRaggedLmin);
        if (b < spec.nb) atomicAdd(&h[b], 1);
        else if (ceil_log2_dev(n) - spec.over_lo >= spec.n_over) atomicAdd(&over, 1);
    }
    __syncthreads();
    if (threadIdx.x < spec.nb && h[threadIdx.x]) atomicAdd(&ctl->count[threadIdx.x], h[threadIdx.x]);
    if (threadIdx.x == 0 && over) atomicAdd(&ctl->too_long, over);
}

// ids[] receives array ids grouped by bucket, largest working length first;
// arrays for the cluster kernels go to their own lists.
__global__ void k_bin_scatter(const int* __restrict__ off, int arrays, RaggedCtl* ctl, int* ids, int* oids,
                              BinSpec spec) {
    const int nb = spec.nb;
    __shared__ int base[kMaxBuckets], h[kMaxBuckets], grab[kMaxBuckets];
    if (threadIdx.x == 0) {
        int s = 0;
        for (int b = nb - 1; b >= 0; --b) {
            base[b] = s;
            if (blockIdx.x == 0) ctl->base[b] = s;  // for the launches of dedicated buckets
            s += ctl->count[b];
        }
    }
    for (int a0 = blockIdx.x * blockDim.x; a0 < arrays; a0 += gridDim.x * blockDim.x) {
        if (threadIdx.x < kMaxBuckets) h[threadIdx.x] = 0;
        __syncthreads();
        const int a = a0 + int(threadIdx.x);
        int b = -1, local = 0;
        if (a < arrays) {
            const int n = off[a + 1] - off[a];
            if (n > 0) {
                b = bucket_of(n, kRaggedLmin);
                if (b < nb) {
                    local = atomicAdd(&h[b], 1);
                } else {
                    const int ob = ceil_log2_dev(n) - spec.over_lo;
                    if (ob < spec.n_over) {
                        const int pos = atomicAdd(&ctl->ocount[ob], 1);
                        oids[size_t(ob) * spec.stride + pos] = a;
                    }
                    b = -1;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x < nb && h[threadIdx.x]) grab[threadIdx.x] = atomicAdd(&ctl->cursor[threadIdx.x], h[threadIdx.x]);
        __syncthreads();
        if (b >= 0) ids[base[b] + grab[b] + local] = a;
        __syncthreads();
    }
}
#else
__global__ void k_bin_count(const int* __restrict__ off, int arrays, RaggedCtl* ctl, BinSpec spec);
__global__ void k_bin_scatter(const int* __restrict__ off, int arrays, RaggedCtl* ctl, int* ids, int* oids,
                              BinSpec spec);
#endif  // B200S_DEFINE_BIN_KERNELS

constexpr int log2_const(int x) { return x <= 1 ? 0 : 1 + log2_const(x / 2); }

// log2 elements per thread of bucket L (= log2 W) in a shape family with
// K = 2^LKF: K elements per thread when a whole team fits the CTA, more when
// it would not (the team never exceeds the CTA).
constexpr int family_lk(int L, int LKF, int LOGCTA) {
    const int lk = L < LKF ? L : LKF;
    return L - lk > LOGCTA ? L - LOGCTA : lk;
}

// Tile of bucket L in a shape family: one lane for W <= K, then more lanes,
// then more warps.
template <int LKF, int L, int CTA>
struct FamilyShape {
    static constexpr int LK = family_lk(L, LKF, log2_const(CTA));
    static constexpr int REST = L - LK;
    static constexpr int LG = REST < 5 ? REST : 5;
    static constexpr int LW = REST - LG;
    using type = Shape<LK, LG, LW>;
};

template <class E, class S, int CTA, bool SB>
__device__ __forceinline__ void ragged_task(const typename E::Mem* in, typename E::Mem* out,
                                            const int* __restrict__ off, const int* __restrict__ ids,
                                            int first_id, int count, int local_task,
                                            unsigned char* smem_raw) {
    using R = typename E::Reg;
    static_assert(CTA % S::TPA == 0, "whole teams per CTA");
    constexpr int APT = CTA / S::TPA;
    const int team = int(threadIdx.x) / S::TPA;
    const int t = int(threadIdx.x) % S::TPA;
    const int idx = local_task * APT + team;
    int na = 0;
    long long start = 0;
    if (idx < count) {
        const int a = ids[first_id + idx];
        start = off[a];
        na = off[a + 1] - off[a];
    }
    R* cur = reinterpret_cast<R*>(smem_raw) + size_t(team) * (SB ? 1 : 2) * S::W;
    R* nxt = SB ? cur : cur + S::W;
    R v[S::K];
    load_tile<E, S::K>(v, in + start, t * S::K, na);
    if constexpr (S::LW > 0) {
        static_assert(CTA / S::TPA <= 15, "named barrier ids");
        if constexpr (SB) network<E, S>(v, t, cur, nxt, TeamBarrierSingle{1 + team, S::TPA}, na);
        else network<E, S>(v, t, cur, nxt, TeamBarrier{1 + team, S::TPA}, na);
    } else {
        network<E, S>(v, t, cur, nxt, CtaBarrier{}, na);
    }
    store_tile<E, S::K>(v, out + start, t * S::K, na);
}

// NB buckets (W = 8 .. 8 << (NB-1)); bucket b uses family B (K = 2^LKB)
// when bit b of family_mask is set, else family A (K = 2^LKA); buckets whose
// bit is set in dedicated_mask are left to their own launches (their ids stay
// in the list at ctl->base[b]).  SB: one shared-memory buffer per team (two
// barriers per shared-memory layer, half the shared memory); MINB: CTAs per
// SM the register budget is sized for.
template <class E, int CTA, int NB, int LKA, int LKB, bool SB, int MINB>
__global__ void __launch_bounds__(CTA, MINB) k_sort_ragged(const typename E::Mem* in, typename E::Mem* out,
                                                        const int* __restrict__ off,
                                                        const int* __restrict__ ids, RaggedCtl* ctl,
                                                        unsigned family_mask, unsigned dedicated_mask) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_first[NB], s_tasks[NB], s_base[NB], s_count[NB];
    __shared__ int s_total, s_task;
    if (threadIdx.x == 0) {
        int task = 0, base = 0;
        for (int b = NB - 1; b >= 0; --b) {
            // dedicated buckets get no tasks here, but their ids still occupy
            // the list, so the bases count them
            const int c = ctl->count[b];
            const int L = b + kRaggedLmin;
            const int lk = family_lk(L, ((family_mask >> b) & 1u) ? LKB : LKA, log2_const(CTA));
            const int tpa = 1 << (L - lk);
            const int apt = CTA / tpa;
            s_first[b] = task;
            s_tasks[b] = ((dedicated_mask >> b) & 1u) ? 0 : (c + apt - 1) / apt;
            s_base[b] = base;
            s_count[b] = c;
            task += s_tasks[b];
            base += c;
        }
        s_total = task;
    }
    __syncthreads();
    const int total = s_total;
    for (;;) {
        if (threadIdx.x == 0) s_task = atomicAdd(&ctl->head, 1);
        __syncthreads();
        const int task = s_task;
        __syncthreads();
        if (task >= total) break;
        int b = NB - 1;
        while (b > 0 && task >= s_first[b] + s_tasks[b]) --b;
        const int local = task - s_first[b];
        const bool fam_b = (family_mask >> b) & 1u;
        sfor<0, NB>([&](auto bc) {
            constexpr int B = decltype(bc)::value;
            constexpr int L = B + kRaggedLmin;
            if (b == B) {
                if (fam_b)
                    ragged_task<E, typename FamilyShape<LKB, L, CTA>::type, CTA, SB>(in, out, off, ids, s_base[B],
                                                                                      s_count[B], local, smem_raw);
                else
                    ragged_task<E, typename FamilyShape<LKA, L, CTA>::type, CTA, SB>(in, out, off, ids, s_base[B],
                                                                                      s_count[B], local, smem_raw);
            }
        });
    }
}

// Shared memory of k_sort_ragged: the largest per-CTA buffer (double, or
// single when SB) over the buckets that use it.
template <class E, int CTA, int NB, int LKA, int LKB, bool SB>
constexpr size_t ragged_smem() {
    size_t best = 0;
    for (int b = 0; b < NB; ++b) {
        const int L = b + kRaggedLmin;
        for (int lkf : {LKA, LKB}) {
            const int k = family_lk(L, lkf, log2_const(CTA));
            const int rest = L - k;
            const int lw = rest > 5 ? rest - 5 : 0;
            if (lw > 0) {
                const size_t bytes = (SB ? 1 : 2) * size_t(CTA) * (size_t(1) << k) * sizeof(typename E::Reg);
                if (bytes > best) best = bytes;
            }
        }
    }
    return best;
}

// Launches over an id list: every array of the list fits the tile; one group
// per array.  With d_count null the grid strides over `count` arrays.
// Otherwise (a dedicated bucket of a ragged plan) the count and the list's
// first position are read on the device, so that a captured launch sorts
// whatever the binning put into its bucket, and the resident CTAs pull groups
// of arrays from the queue at d_head (one atomicAdd per group), which keeps
// them busy when the arrays' lengths, and so their costs, differ.
template <class E, class S, int CTA, bool SB = false>
__global__ void __launch_bounds__(CTA) k_sort_idlist(const typename E::Mem* in, typename E::Mem* out,
                                                     const int* __restrict__ off, const int* __restrict__ ids,
                                                     int count, const int* d_count, const int* d_base,
                                                     int* d_head) {
    using R = typename E::Reg;
    __shared__ int s_next;
    if (d_count) {
        count = *d_count;
        ids += *d_base;
    }
    constexpr int APC = CTA / S::TPA;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* cur = reinterpret_cast<R*>(smem_raw);
    R* nxt = SB ? cur : cur + S::W;  // the launch passes 1 or 2 buffers of W elements
    const int slot = int(threadIdx.x) / S::TPA;
    const int t = int(threadIdx.x) % S::TPA;
    long long first = (long long)blockIdx.x * APC;
    for (;;) {
        if (d_head) {
            if (threadIdx.x == 0) s_next = atomicAdd(d_head, APC);
            __syncthreads();
            first = s_next;
            __syncthreads();
        }
        if (first >= count) break;  // uniform across the CTA
        const long long g = first + slot;
        int na = 0;
        long long start = 0;
        if (g < count) {
            const int a = ids[g];
            start = off[a];
            na = off[a + 1] - off[a];
        }
        R v[S::K];
        load_tile<E, S::K>(v, in + start, t * S::K, na);
        if constexpr (SB) network<E, S>(v, t, cur, nxt, CtaBarrierSingle{}, na);
        else network<E, S>(v, t, cur, nxt, CtaBarrier{}, na);
        store_tile<E, S::K>(v, out + start, t * S::K, na);
        if (!d_head) first += (long long)gridDim.x * APC;
    }
}

}  // namespace b200s
