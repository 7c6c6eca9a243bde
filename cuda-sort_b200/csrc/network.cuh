// The reflection bitonic network, mapped onto registers, warp lanes and
// shared memory of one B200 CTA.
//
// Network (same comparators as cusort_v6.hpp:90-142): for each stage span
// S = 1, 2, ..., W/2, one reflection layer pairing index i with i ^ (2S-1),
// then merge layers pairing i with i ^ d for d = S/2, ..., 1.  In every pair
// the lower index receives the smaller element, and an exchange happens only
// when the upper element is strictly smaller (the keep-own rule of
// cusort.hpp:460-472).  Because of that rule, maximum-key padding placed after
// the n valid elements never moves, so any power-of-two W >= n yields the
// same output; the tile table is free to choose W.
//
// Mapping (blocked): the W-element working tile is held as K = 2^LK
// consecutive elements per thread.  Index bits [0, LK) select a register,
// bits [LK, LK+LG) a lane inside a group of G = 2^LG lanes, and bits
// [LK+LG, LK+LG+LW) a warp.  A layer whose highest flipped bit is a register
// bit is a compare-exchange between two registers of the same thread; a lane
// bit makes it one __shfl_xor_sync per element; a warp bit makes it one
// shared-memory publish + read per element, double-buffered so that each such
// layer costs a single __syncthreads.  With K = 32 and a warp per 1024-key
// array, 40 of the 55 layers run in registers and 15 on the shuffle unit;
// none touches shared memory.
#pragma once
#include <cstdint>
#include <type_traits>

#include "elem.cuh"
#include "opts.h"

namespace b200s {

template <int I, int N, class F>
__device__ __forceinline__ void sfor(F&& f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        sfor<I + 1, N>(f);
    }
}

// Barrier over the threads that share one array's shared-memory tile: the
// whole CTA when an array owns its CTA, or a named barrier when several
// multi-warp teams share a CTA (ids 1..15; id 0 is __syncthreads).
// unaligned(): the same barrier for warps that reach it from different code
// (barrier.sync without .aligned): the compact network runs warps of padding
// through a copy of the layer sequence that only publishes and synchronises.
struct CtaBarrier {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
    __device__ __forceinline__ void unaligned() const { asm volatile("barrier.sync 0;" ::: "memory"); }
};
// __syncthreads with one shared-memory buffer (see single_buffer below).
struct CtaBarrierSingle {
    static constexpr bool kSingleBuffer = true;
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
    __device__ __forceinline__ void unaligned() const { asm volatile("barrier.sync 0;" ::: "memory"); }
};
struct TeamBarrier {
    int id;
    int threads;
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
    }
    __device__ __forceinline__ void unaligned() const {
        asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
    }
};
// The same with one shared-memory buffer per team (see single_buffer below).
struct TeamBarrierSingle {
    static constexpr bool kSingleBuffer = true;
    int id;
    int threads;
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
    }
    __device__ __forceinline__ void unaligned() const {
        asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
    }
};

constexpr int hibit(unsigned x) {
    int b = -1;
    while (x) {
        x >>= 1;
        ++b;
    }
    return b;
}

template <int LK_, int LG_, int LW_>
struct Shape {
    static constexpr int LK = LK_, LG = LG_, LW = LW_;
    static constexpr int K = 1 << LK;          // elements per thread
    static constexpr int G = 1 << LG;          // lanes per array inside a warp
    static constexpr int TPA = G << LW;        // threads per array
    static constexpr int LOGW = LK + LG + LW;
    static constexpr int W = 1 << LOGW;        // working tile length
    static_assert(LG >= 0 && LG <= 5, "lane bits");
    static_assert(LW == 0 || LG == 5, "an array spanning warps uses whole warps");
};

// Barrier policies may set kSingleBuffer: then a shared-memory layer publishes
// into one buffer and synchronises again after reading it (two barriers, half
// the shared memory); otherwise it alternates two buffers with one barrier.
template <class Bar, class = void>
struct single_buffer : std::false_type {};
template <class Bar>
struct single_buffer<Bar, std::void_t<decltype(Bar::kSingleBuffer)>>
    : std::integral_constant<bool, Bar::kSingleBuffer> {};

// One comparator layer with partner mask MASK (compile-time).
template <class E, class S, unsigned MASK, class Bar>
__device__ __forceinline__ void layer(typename E::Reg (&v)[S::K], const int t,
                                      typename E::Reg*& cur, typename E::Reg*& nxt, const Bar& bar) {
    using R = typename E::Reg;
    constexpr int HB = hibit(MASK);
    constexpr unsigned RM = MASK & unsigned(S::K - 1);
    constexpr unsigned TM = MASK >> S::LK;
    if constexpr (HB < S::LK) {
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr int p = q ^ int(MASK);
            if constexpr (q < p) E::cex(v[q], v[p]);
        });
    } else if constexpr (HB < S::LK + S::LG) {
        const bool upper = (t >> (HB - S::LK)) & 1;
        if constexpr (RM == 0) {
            sfor<0, S::K>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                const R b = E::shfl(v[q], int(TM));
                v[q] = E::pick(v[q], b, upper);
            });
        } else {
            // Reflection across lanes: the partner of (lane, q) is
            // (lane ^ TM, q ^ RM).  Exchange both registers of a pair before
            // updating either.
            sfor<0, S::K>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                constexpr int p = q ^ int(RM);
                if constexpr (q < p) {
                    const R bq = E::shfl(v[p], int(TM));
                    const R bp = E::shfl(v[q], int(TM));
                    v[q] = E::pick(v[q], bq, upper);
                    v[p] = E::pick(v[p], bp, upper);
                }
            });
        }
    } else {
        const bool upper = (t >> (HB - S::LK)) & 1;
        // Striped publication: register q of every thread forms one row, so
        // both the publish and the partner read are bank-conflict free.
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            sh_st(&cur[q * S::TPA + t], v[q]);
        });
        bar();
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const R b = sh_ld(&cur[(q ^ int(RM)) * S::TPA + (t ^ int(TM))]);
            v[q] = E::pick(v[q], b, upper);
        });
        if constexpr (single_buffer<Bar>::value) {
            bar();
        } else {
            R* tmp = cur;
            cur = nxt;
            nxt = tmp;
        }
    }
}

template <class E, class S, int ST, class Bar>
__device__ __forceinline__ void stage(typename E::Reg (&v)[S::K], const int t,
                                      typename E::Reg*& cur, typename E::Reg*& nxt, const Bar& bar) {
    layer<E, S, (2u << ST) - 1u>(v, t, cur, nxt, bar);   // reflection, span 2^ST
    sfor<0, ST>([&](auto jc) {
        constexpr int j = ST - 1 - decltype(jc)::value;
        layer<E, S, (1u << j)>(v, t, cur, nxt, bar);       // merges 2^(ST-1) .. 1
    });
}

// ---- compact form ------------------------------------------------------------
// The same layers with the lane / warp part of the partner mask known only at
// run time, so that the stages whose span leaves the registers share one copy
// of their code.  A cross-lane or cross-warp layer pairs (t, q) with
// (t ^ tm, q ^ RM): RM is all register bits for a reflection and 0 for a
// merge, whatever the stage.

template <class E, class S, unsigned RM>
__device__ __forceinline__ void lane_layer_rt(typename E::Reg (&v)[S::K], const int tm, const bool upper) {
    using R = typename E::Reg;
    if constexpr (RM == 0) {
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const R b = E::shfl(v[q], tm);
            v[q] = E::pick(v[q], b, upper);
        });
    } else {
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr int p = q ^ int(RM);
            if constexpr (q < p) {
                const R bq = E::shfl(v[p], tm);
                const R bp = E::shfl(v[q], tm);
                v[q] = E::pick(v[q], bq, upper);
                v[p] = E::pick(v[p], bp, upper);
            }
        });
    }
}

// LIVE == false: the copy run by a warp that holds only padding: it still
// publishes (its partners read it) and meets every barrier, but compares
// nothing.  Both copies take the same barriers in the same order.
// UA: unaligned barriers, for teams whose warps run different copies.
template <class E, class S, unsigned RM, bool LIVE, bool UA, class Bar>
__device__ __forceinline__ void warp_layer_rt(typename E::Reg (&v)[S::K], const int t, const int tm,
                                              const bool upper, typename E::Reg*& cur, typename E::Reg*& nxt,
                                              const Bar& bar) {
    using R = typename E::Reg;
    sfor<0, S::K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        sh_st(&cur[q * S::TPA + t], v[q]);
    });
    if constexpr (UA) bar.unaligned();
    else bar();
    if constexpr (LIVE) {
        sfor<0, S::K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const R b = sh_ld(&cur[(q ^ int(RM)) * S::TPA + (t ^ tm)]);
            v[q] = E::pick(v[q], b, upper);
        });
    }
    if constexpr (single_buffer<Bar>::value) {
        if constexpr (UA) bar.unaligned();
        else bar();
    } else {
        R* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
}

// Layer with partner mask bit j >= LK (runtime j); reflection when RM != 0.
template <class E, class S, unsigned RM, bool LIVE, bool UA, class Bar>
__device__ __forceinline__ void cross_layer_rt(typename E::Reg (&v)[S::K], const int t, const int j,
                                               typename E::Reg*& cur, typename E::Reg*& nxt, const Bar& bar) {
    const int tm = RM ? (2 << (j - S::LK)) - 1 : 1 << (j - S::LK);
    const bool upper = (t >> (j - S::LK)) & 1;
    if constexpr (S::LW == 0) {
        if constexpr (LIVE) lane_layer_rt<E, S, RM>(v, tm, upper);
    } else {
        if (j < S::LK + S::LG) {
            if constexpr (LIVE) lane_layer_rt<E, S, RM>(v, tm, upper);
        } else {
            warp_layer_rt<E, S, RM, LIVE, UA>(v, t, tm, upper, cur, nxt, bar);
        }
    }
}

// LIVE == false is the copy for a warp of a multi-warp team whose elements
// are all padding (index >= n).  Padding is the maximum element and never
// moves, so every comparator among padding elements is a no-op and every
// comparator of a real element with padding leaves both in place: such a
// warp skips all its register and lane layers and only takes part in the
// shared-memory exchanges (publish + the same barriers in the same order).
// The output is unchanged, bit for bit.  UA: the team's warps run different
// copies, so its barriers are the unaligned form; a team without padding
// warps runs the LIVE copy with the aligned barriers.
template <class E, class S, bool LIVE, bool UA, class Bar>
__device__ __forceinline__ void network_compact(typename E::Reg (&v)[S::K], const int t, typename E::Reg*& cur,
                                                typename E::Reg*& nxt, const Bar& bar) {
    constexpr int LK = S::LK;
    // stages inside the registers: unrolled
    if constexpr (LIVE)
        sfor<0, (LK < S::LOGW ? LK : S::LOGW)>([&](auto sc) { stage<E, S, decltype(sc)::value>(v, t, cur, nxt, bar); });
#pragma unroll 1
    for (int st = LK; st < S::LOGW; ++st) {
        cross_layer_rt<E, S, unsigned(S::K - 1), LIVE, UA>(v, t, st, cur, nxt, bar);  // reflection
#pragma unroll 1
        for (int j = st - 1; j >= LK; --j) cross_layer_rt<E, S, 0u, LIVE, UA>(v, t, j, cur, nxt, bar);
        // merges 2^(LK-1) .. 1 inside the registers
        if constexpr (LIVE) {
            sfor<0, LK>([&](auto jc) {
                constexpr int j = LK - 1 - decltype(jc)::value;
                layer<E, S, (1u << j)>(v, t, cur, nxt, bar);
            });
        }
    }
}

// The unrolled form is kept where its code stays small (a compare-exchange
// of int32 keys is two instructions, E::kCompact false); the other element
// types take several instructions per compare-exchange and their fully
// unrolled networks overflow the instruction cache, so they use the compact
// form.
template <class E, class S>
constexpr bool use_compact() {
    return E::kCompact && S::LOGW > S::LK;
}

// Whether the warp of team thread t holds any element below n: false only
// for whole warps of padding in a team of whole warps (teams smaller than a
// warp share it with other arrays and always count as live).
template <class S>
__device__ __forceinline__ bool warp_live(const int t, const long long n, const long long first = 0) {
    if constexpr (S::LG == 5) return first + (long long)(t >> 5) * (32 * S::K) < n;
    else return true;
}

// Sort the W-element tile held by the TPA threads of one array of n
// elements.  The compact form runs warps of padding through the copy that
// only publishes and synchronises (see network_compact); the unrolled form,
// kept for int32 keys, runs every warp through the whole network.
template <class E, class S, class Bar = CtaBarrier>
__device__ __forceinline__ void network(typename E::Reg (&v)[S::K], const int t,
                                        typename E::Reg*& cur, typename E::Reg*& nxt,
                                        const Bar& bar = Bar(), const long long n = S::W) {
    if constexpr (use_compact<E, S>()) {
        if constexpr (S::LW <= 1) {
            // At most two warps: a warp of padding would need n <= W/2, for
            // which a tile of half the width is chosen.
            network_compact<E, S, true, false>(v, t, cur, nxt, bar);
        } else {
            if (warp_live<S>(S::TPA - 1, n)) network_compact<E, S, true, false>(v, t, cur, nxt, bar);
            else if (warp_live<S>(t, n)) network_compact<E, S, true, true>(v, t, cur, nxt, bar);
            else network_compact<E, S, false, true>(v, t, cur, nxt, bar);
        }
    } else {
        sfor<0, S::LOGW>([&](auto sc) { stage<E, S, decltype(sc)::value>(v, t, cur, nxt, bar); });
    }
}

// ---- tile load / store --------------------------------------------------------
// Thread t of an array owns elements [t*K, t*K+K).  Whole, 16-byte aligned
// spans move as 128-bit accesses; a ragged tail or an unaligned array start
// falls back to one access per element.  Elements at or beyond n are padding.
template <class E, int K>
__device__ __forceinline__ void load_tile(typename E::Reg (&v)[K], const typename E::Mem* src,
                                          const int base, const int n) {
    using M = typename E::Mem;
    constexpr int BYTES = K * int(sizeof(M));
    if constexpr (BYTES % 16 == 0) {
        if (base + K <= n && (reinterpret_cast<uintptr_t>(src + base) & 15u) == 0) {
            constexpr int PER = 16 / int(sizeof(M));
            const uint4* p = reinterpret_cast<const uint4*>(src + base);
            sfor<0, BYTES / 16>([&](auto cc) {
                constexpr int c = decltype(cc)::value;
                const uint4 u = __ldcs(p + c);
                sfor<0, PER>([&](auto jc) {
                    constexpr int j = decltype(jc)::value;
                    M m;
                    from_u4<j>(u, m);
                    v[c * PER + j] = E::from_mem(m, base + c * PER + j);
                });
            });
            return;
        }
    }
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const int idx = base + q;
        v[q] = idx < n ? E::from_mem(src[idx], idx) : E::pad();
    }
}

template <class E, int K>
__device__ __forceinline__ void store_tile(const typename E::Reg (&v)[K], typename E::Mem* dst,
                                           const int base, const int n) {
    using M = typename E::Mem;
    constexpr int BYTES = K * int(sizeof(M));
    if constexpr (BYTES % 16 == 0) {
        if (base + K <= n && (reinterpret_cast<uintptr_t>(dst + base) & 15u) == 0) {
            constexpr int PER = 16 / int(sizeof(M));
            uint4* p = reinterpret_cast<uint4*>(dst + base);
            sfor<0, BYTES / 16>([&](auto cc) {
                constexpr int c = decltype(cc)::value;
                uint4 u;
                sfor<0, PER>([&](auto jc) {
                    constexpr int j = decltype(jc)::value;
                    to_u4<j>(u, E::to_mem(v[c * PER + j]));
                });
                __stcs(p + c, u);
            });
            return;
        }
    }
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const int idx = base + q;
        if (idx < n) dst[idx] = E::to_mem(v[q]);
    }
}

// ---- sortedness check (the reference's Sorted switch) -------------------------
// With its Sorted switch the reference tests the tile before the first stage
// (and after every stage of span >= 16) and returns early when the tile is
// already in order (cusort_v6.hpp:103-128, cusort.hpp:437-458).  A tile in
// order is a fixed point of every comparator under the keep-own rule, so the
// early return changes no output.  Padding (the maximum element after the n
// valid ones) never breaks the order, so the whole tile is tested.

template <class E, int K>
__device__ __forceinline__ bool thread_in_order(const typename E::Reg (&v)[K]) {
    bool ok = true;
    sfor<0, K - 1>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        ok &= !E::after(v[q], v[q + 1]);
    });
    return ok;
}

// Whether the tile of team thread t (blocked layout, TPA threads) is in order.
// The answer is uniform where the network needs it: over the CTA for a
// multi-warp team (one array per CTA), over the warp for teams inside a warp
// (true only when every array of the warp is in order), so that every lane
// of a warp and every warp of a CTA takes the same branch.  cur: the team's
// shared buffer (free before the network), used for the warp boundaries.
template <class E, class S>
__device__ __forceinline__ bool team_in_order(const typename E::Reg (&v)[S::K], const int t,
                                              typename E::Reg* cur) {
    using R = typename E::Reg;
    bool ok = thread_in_order<E, S::K>(v);
    const R nx = E::shfl_down(v[0], 1);  // the next lane's first element
    const bool last_of_group = ((t + 1) & (S::G - 1)) == 0;
    if (!last_of_group) ok &= !E::after(v[S::K - 1], nx);
    if constexpr (S::LW == 0) {
        return __all_sync(0xffffffffu, ok);
    } else {
        const int lane = t & 31, w = t >> 5;
        if (lane == 0) cur[w] = v[0];
        __syncthreads();
        if (lane == 31 && w + 1 < (S::TPA >> 5)) ok &= !E::after(v[S::K - 1], cur[w + 1]);
        return __syncthreads_and(ok) != 0;
    }
}

// ---- packed batch kernel ------------------------------------------------------
// Packed layout of the reference's batched wrappers (bench.cu:355-393):
// array a occupies [a*n, a*n + n).  Each group of TPA threads sorts one array;
// a CTA holds CTA/TPA groups and strides over the batch.  The loop bound is
// uniform across the CTA, so groups past the end sort padding and store
// nothing, and every warp-wide shuffle and barrier sees all its threads.
// SB: one shared-memory buffer (two barriers per shared-memory layer, half the
// shared memory, more CTAs per SM) instead of two.
// opts & kOptSortedCheck: test each tile first and skip the network when it is
// already in order (and the store too when sorting in place).
template <class E, class S, int CTA, bool SB = false>
__global__ void __launch_bounds__(CTA) k_sort_packed(const typename E::Mem* in,
                                                     typename E::Mem* out, int n,
                                                     long long arrays, unsigned opts) {
    using R = typename E::Reg;
    static_assert(CTA % S::TPA == 0, "CTA holds whole arrays");
    static_assert(S::LW == 0 || CTA == S::TPA, "a multi-warp array owns its CTA");
    constexpr int APC = CTA / S::TPA;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* cur = reinterpret_cast<R*>(smem_raw);
    R* nxt = SB ? cur : cur + S::W;
    const int slot = int(threadIdx.x) / S::TPA;
    const int t = int(threadIdx.x) % S::TPA;
    // programmatic dependent launch: wait for the stream's previous kernel
    // (immediate when launched without the attribute), then release the next
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    for (long long first = (long long)blockIdx.x * APC; first < arrays;
         first += (long long)gridDim.x * APC) {
        const long long a = first + slot;
        const int na = a < arrays ? n : 0;
        const long long off = (a < arrays ? a : 0) * (long long)n;
        R v[S::K];
        load_tile<E, S::K>(v, in + off, t * S::K, na);
        const bool skip = (opts & kOptSortedCheck) && team_in_order<E, S>(v, t, cur);
        if (!skip) {
            if constexpr (SB) network<E, S>(v, t, cur, nxt, CtaBarrierSingle{}, na);
            else network<E, S>(v, t, cur, nxt, CtaBarrier{}, na);
        }
        if (!skip || in != out) store_tile<E, S::K>(v, out + off, t * S::K, na);
    }
}

// Persistent form: the grid is sized to the resident capacity and each group
// walks the batch with a stride of the whole grid, loading the next array's
// tile into registers before sorting the current one, so that the global
// loads of one array overlap the comparator layers of the previous one.
template <class E, class S, int CTA, bool SB = false>
__global__ void __launch_bounds__(CTA) k_sort_packed_pf(const typename E::Mem* in,
                                                        typename E::Mem* out, int n,
                                                        long long arrays, unsigned opts) {
    using R = typename E::Reg;
    constexpr int APC = CTA / S::TPA;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* cur = reinterpret_cast<R*>(smem_raw);
    R* nxt = SB ? cur : cur + S::W;
    const int slot = int(threadIdx.x) / S::TPA;
    const int t = int(threadIdx.x) % S::TPA;
    const long long stride = (long long)gridDim.x * APC;
    long long first = (long long)blockIdx.x * APC;
    // programmatic dependent launch (see k_sort_packed)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (first >= arrays) return;  // uniform across the CTA
    R v[S::K];
    {
        const long long a = first + slot;
        load_tile<E, S::K>(v, in + (a < arrays ? a : 0) * (long long)n, t * S::K, a < arrays ? n : 0);
    }
    for (; first < arrays; first += stride) {
        const long long a = first + slot;
        const long long an = a + stride;
        R w[S::K];
        load_tile<E, S::K>(w, in + (an < arrays ? an : 0) * (long long)n, t * S::K, an < arrays ? n : 0);
        const bool skip = (opts & kOptSortedCheck) && team_in_order<E, S>(v, t, cur);
        if (!skip) {
            if constexpr (SB) network<E, S>(v, t, cur, nxt, CtaBarrierSingle{}, a < arrays ? n : 0);
            else network<E, S>(v, t, cur, nxt, CtaBarrier{}, a < arrays ? n : 0);
        }
        if (a < arrays && (!skip || in != out)) store_tile<E, S::K>(v, out + a * (long long)n, t * S::K, n);
#pragma unroll
        for (int q = 0; q < S::K; ++q) v[q] = w[q];
    }
}

}  // namespace b200s
