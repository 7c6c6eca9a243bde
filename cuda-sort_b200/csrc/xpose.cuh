// The reflection bitonic network with every comparator layer in registers:
// launch form 3 ("transposed network") of one-warp-or-smaller tiles.
//
// The network is the one of cusort_v6.hpp:90-142 (see network.cuh): for each
// stage ST, a reflection layer pairing i with i ^ (2^(ST+1) - 1), then merges
// pairing i with i ^ 2^j, j = ST-1 .. 0, lower index takes the minimum, and an
// exchange happens only on a strict `<` (keep-own, cusort.hpp:460-472).
//
// Mapping.  A tile of W = K * G elements (K = 2^LK per thread, G = 2^LG lanes
// per array, LK + LG <= 2 LK) is held by G lanes.  In the natural layout lane
// t holds logical indices [t*K, t*K + K): index bits [0, LK) are register
// bits, so stages 0 .. LK-1 run in registers as in network.cuh.  For a later
// stage ST the tile is re-laid out twice through a per-array shared-memory
// region, so that every layer is a compare-exchange between two registers of
// one thread (never a shuffle, whose one-sided min/max costs two ALU
// instructions per element instead of one):
//   1. natural -> window layout W_ST: register bit r holds index bit
//      ST-LK+1+r (the LK bits ST-LK+1 .. ST), lanes hold the others;
//      registers whose index bit ST is set (the upper half of each 2^(ST+1)
//      block) read the MIRRORED element: its index bits below ST complemented.
//      Then the reflection partner of register q (upper bit clear) is register
//      q + K/2: a plain register pair.  Inside the mirrored half a merge's
//      lower logical index sits in the physically upper register, so those
//      merges put the minimum into the upper register; both choices are
//      compile-time.  Reflection + merges on bits ST-1 .. ST-LK+1 run here.
//   2. window -> natural (the shared region stores element i at its logical
//      address, so reading it back un-mirrors it); merges on bits ST-LK .. 0
//      run in registers.
// Each comparator compares the same two elements as the reference's network,
// with the same keep-own rule, so the output (tie order of records included)
// is the reference's.
//
// Shared-memory layout: element of logical index i at xp_addr(i) = i + (i >>
// LK), one pad element per K.  Every index bit then contributes a power of two
// modulo 32 banks, and in every layout above the lane bits of an array hit
// distinct powers (their weights are 2^0 .. 2^(LG-1) up to order); so each
// 32-bit access instruction is conflict-free, and the regions of the 32/G
// arrays of a warp, W + G elements apart (= G modulo 32), fill the other
// banks.  Addresses are a per-lane base (three per stage: natural, window,
// mirrored window) plus a compile-time offset per register: the transposes
// cost no ALU instructions beyond a few per stage and lane.
#pragma once
#include <cstdint>
#include <type_traits>

#include "network.cuh"

namespace b200s {

// Compare-exchange number Q of a layer.  An element type with kFmaSplit runs
// two of every three in its cex_fma form, which leaves the minimum on the ALU
// pipe and forms the maximum as a + b - min with two integer multiply-adds on
// the FMA pipe (exact in two's complement), so both pipes share the layer.
template <class E, class = void>
struct fma_split : std::false_type {};
template <class E>
struct fma_split<E, std::void_t<decltype(E::kFmaSplit)>> : std::integral_constant<bool, E::kFmaSplit> {};

template <class E, class = void>
struct fma_period : std::integral_constant<int, 3> {};
template <class E>
struct fma_period<E, std::void_t<decltype(E::kFmaPeriod)>> : std::integral_constant<int, E::kFmaPeriod> {};

template <class E, int Q>
__device__ __forceinline__ void xcex(typename E::Reg& lo, typename E::Reg& hi) {
    constexpr int P = fma_period<E>::value;  // P > 0: one in P in the FMA form; P < 0: all but one in -P
    if constexpr (fma_split<E>::value && (P > 0 ? (Q % P) == 0 : (Q % -P) != 0)) E::cex_fma(lo, hi);
    else E::cex(lo, hi);
}

// Streaming (evict-first) global accesses of one element of each memory
// layout; records move as one 8- or 16-byte access, so their arrays must be
// aligned to the record size (the C ABI checks before choosing this form).
__device__ __forceinline__ int32_t xp_ldcs(const int32_t* p) { return __ldcs(p); }
__device__ __forceinline__ uint64_t xp_ldcs(const uint64_t* p) {
    return __ldcs(reinterpret_cast<const unsigned long long*>(p));
}
__device__ __forceinline__ RecI32 xp_ldcs(const RecI32* p) {
    const int2 v = __ldcs(reinterpret_cast<const int2*>(p));
    return RecI32{v.x, v.y};
}
__device__ __forceinline__ void xp_stcs(int32_t* p, int32_t v) { __stcs(p, v); }
__device__ __forceinline__ void xp_stcs(uint64_t* p, uint64_t v) {
    __stcs(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
__device__ __forceinline__ void xp_stcs(RecI32* p, RecI32 v) { __stcs(reinterpret_cast<int2*>(p), make_int2(v.key, v.data)); }

// Element types whose tie order cannot be observed (keys alone: equal keys
// are indistinguishable) may sort a thread's registers with any network that
// leaves them in ascending order; records keep the reflection network.
template <class E, class = void>
struct keys_only : std::false_type {};
template <class E>
struct keys_only<E, std::void_t<decltype(E::kKeysOnly)>> : std::integral_constant<bool, E::kKeysOnly> {};

// Batcher's odd-even merge sort of N = 2^L registers, in its published
// iterative form (for p = 1, 2, 4, ...; k = p, p/2, ..., 1; j = k mod p,
// j + 2k, ...; i < k: compare j+i with j+i+k when both lie in the same block
// of 2p): the lower index receives the minimum.  Same depth as the bitonic
// sort, fewer comparators (191 instead of 240 for 32 registers, 63 instead of
// 80 for 16), and the same result for keys: the registers end sorted, as
// after stages 0 .. L-1 of the reflection network.
template <int N>
struct OddEvenMergeSort {
    struct Pair {
        int a, b;
    };
    static constexpr int count() {
        int c = 0;
        for (int p = 1; p < N; p *= 2)
            for (int k = p; k >= 1; k /= 2)
                for (int j = k % p; j <= N - 1 - k; j += 2 * k)
                    for (int i = 0; i <= k - 1 && i <= N - j - k - 1; ++i)
                        if ((i + j) / (2 * p) == (i + j + k) / (2 * p)) ++c;
        return c;
    }
    struct Table {
        Pair pairs[count()];
    };
    static constexpr Table table() {
        Table t{};
        int c = 0;
        for (int p = 1; p < N; p *= 2)
            for (int k = p; k >= 1; k /= 2)
                for (int j = k % p; j <= N - 1 - k; j += 2 * k)
                    for (int i = 0; i <= k - 1 && i <= N - j - k - 1; ++i)
                        if ((i + j) / (2 * p) == (i + j + k) / (2 * p)) t.pairs[c++] = Pair{i + j, i + j + k};
        return t;
    }
    static constexpr Table kTable = table();
};

template <class E, int LK>
__device__ __forceinline__ void xp_reg_sort_oem(typename E::Reg (&v)[1 << LK]) {
    using T = OddEvenMergeSort<(1 << LK)>;
    sfor<0, T::count()>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        constexpr int a = T::kTable.pairs[i].a, b = T::kTable.pairs[i].b;
        xcex<E, i>(v[a], v[b]);
    });
}

template <int LK>
__host__ __device__ constexpr int xp_addr(int i) {
    return i + (i >> LK);
}

// Offset of register q in the window layout of stage ST (upper half mirrored).
template <int LK, int ST>
__host__ __device__ constexpr int xp_win_off(int q) {
    constexpr int H = (1 << LK) >> 1;
    return xp_addr<LK>(((q & H) ? (q ^ (H - 1)) : q) << (ST - LK + 1));
}

template <class E, int LK, int LG, int ST>
__device__ __forceinline__ void xp_stage(typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm) {
    constexpr int K = 1 << LK, H = K >> 1;
    constexpr int LOW = ST - LK + 1;  // lane bits below the window: index bits 0 .. LOW-1
    constexpr int LOWMASK = (1 << LOW) - 1;
    static_assert(LOW >= 1 && LOW <= LG, "stage outside the two-window range");
    const int hi = (t >> LOW) << (ST + 1);
    const int lo = t & LOWMASK;
    const int bp = xp_addr<LK>(hi | lo);              // window, lower half
    const int bm = xp_addr<LK>(hi | (lo ^ LOWMASK));  // window, mirrored upper half
    const int bn = xp_addr<LK>(t << LK);              // natural
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        sm[bn + xp_addr<LK>(q)] = v[q];
    });
    __syncwarp();
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        v[q] = sm[((q & H) ? bm : bp) + xp_win_off<LK, ST>(q)];
    });
    __syncwarp();
    // reflection: register q with its mirror partner q + K/2
    sfor<0, H>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        xcex<E, q>(v[q], v[q + H]);
    });
    // merges on index bits ST-1 .. ST-LK+1 = register bits LK-2 .. 0
    sfor<0, LK - 1>([&](auto rc) {
        constexpr int r = LK - 2 - decltype(rc)::value;
        sfor<0, K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (!(q & (1 << r))) {
                if constexpr (q & H) xcex<E, q>(v[q | (1 << r)], v[q]);  // mirrored: minimum goes up
                else xcex<E, q>(v[q], v[q | (1 << r)]);
            }
        });
    });
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        sm[((q & H) ? bm : bp) + xp_win_off<LK, ST>(q)] = v[q];
    });
    __syncwarp();
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        v[q] = sm[bn + xp_addr<LK>(q)];
    });
    __syncwarp();
    // merges on index bits LOW-1 .. 0 (natural layout: register bits)
    sfor<0, LOW>([&](auto jc) {
        constexpr int j = LOW - 1 - decltype(jc)::value;
        sfor<0, K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (!(q & (1 << j))) xcex<E, q>(v[q], v[q | (1 << j)]);
        });
    });
}

// Stage ST < LK: every layer inside one thread's registers (reflection
// q ^ (2^(ST+1) - 1), then merges q ^ 2^j).
template <class E, int LK, int ST>
__device__ __forceinline__ void xp_reg_stage(typename E::Reg (&v)[1 << LK]) {
    constexpr int K = 1 << LK;
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int p = q ^ ((2 << ST) - 1);
        if constexpr (q < p) xcex<E, q>(v[q], v[p]);
    });
    sfor<0, ST>([&](auto jc) {
        constexpr int j = ST - 1 - decltype(jc)::value;
        sfor<0, K>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (!(q & (1 << j))) xcex<E, q>(v[q], v[q | (1 << j)]);
        });
    });
}

// Whether every array of the warp is in order (natural layout, G lanes per
// array): warp-uniform, since the stages use full-warp synchronisation.
template <class E, int LK, int LG>
__device__ __forceinline__ bool xp_warp_in_order(const typename E::Reg (&v)[1 << LK], const int t) {
    constexpr int K = 1 << LK, G = 1 << LG;
    bool ok = thread_in_order<E, K>(v);
    const typename E::Reg nx = E::shfl_down(v[0], 1);
    if (t != G - 1) ok &= !E::after(v[K - 1], nx);
    return __all_sync(0xffffffffu, ok);
}

// Sort the W = 2^(LK+LG) element tile of lane t (natural layout in and out).
// check: the reference's Sorted switch: after every stage of span >= 16
// (stage index >= 4) stop as soon as every array of the warp is in order.
template <class E, int LK, int LG>
__device__ __forceinline__ void xp_network(typename E::Reg (&v)[1 << LK], const int t, typename E::Reg* sm,
                                           const bool check = false) {
    bool done = false;
    if constexpr (keys_only<E>::value) {
        xp_reg_sort_oem<E, LK>(v);  // stages 0 .. LK-1 with fewer comparators
        if (LK >= 5 && check) done = xp_warp_in_order<E, LK, LG>(v, t);
    } else {
        sfor<0, LK>([&](auto sc) {
            constexpr int ST = decltype(sc)::value;
            if (!done) {
                xp_reg_stage<E, LK, ST>(v);
                if (ST >= 4 && check) done = xp_warp_in_order<E, LK, LG>(v, t);
            }
        });
    }
    sfor<LK, LK + LG>([&](auto sc) {
        constexpr int ST = decltype(sc)::value;
        if (!done) {
            xp_stage<E, LK, LG, ST>(v, t, sm);
            if (check && ST + 1 < LK + LG) done = xp_warp_in_order<E, LK, LG>(v, t);
        }
    });
}

template <int LK, int LG>
constexpr int xp_region() {
    return (1 << (LK + LG)) + (1 << LG);  // W + W / K elements
}

// Coalesced tile access for element types whose input order is unobservable
// (keys alone: equal keys are indistinguishable, so any permutation of an
// array sorts to the same output).  Lane t of a G-lane team reads elements
// t, t + G, t + 2G, ... (one 128-byte wavefront per warp instruction for
// 4-byte keys and G = 32) and calls them its natural-layout registers 0 .. K-1:
// a relabelling of the input, not a data movement.  Elements at or beyond n
// are padding.
template <class E, int LK, int LG>
__device__ __forceinline__ void xp_load_striped(typename E::Reg (&v)[1 << LK], const typename E::Mem* src,
                                                const int t, const int n) {
    constexpr int K = 1 << LK, G = 1 << LG;
    if (n == K * G) {
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] = E::from_mem(xp_ldcs(src + q * G + t), q * G + t);
    } else {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const int idx = q * G + t;
            v[q] = idx < n ? E::from_mem(xp_ldcs(src + idx), idx) : E::pad();
        }
    }
}

// Coalesced load that keeps the input order (any element type): lane t reads
// elements t, t + G, ... (for 8-byte records one 256-byte row per warp
// instruction), writes each at its logical address in the shared region, and
// reads its natural-layout registers [t*K, t*K + K) back; conflict-free like
// the store below.  Elements at or beyond n are padding.
template <class E, int LK, int LG>
__device__ __forceinline__ void xp_load_staged(typename E::Reg (&v)[1 << LK], const typename E::Mem* src,
                                               const int t, const int n, typename E::Reg* sm) {
    constexpr int K = 1 << LK, G = 1 << LG;
    if (n == K * G) {
#pragma unroll
        for (int q = 0; q < K; ++q) sm[xp_addr<LK>(q * G + t)] = E::from_mem(xp_ldcs(src + q * G + t), q * G + t);
    } else {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const int idx = q * G + t;
            sm[xp_addr<LK>(idx)] = idx < n ? E::from_mem(xp_ldcs(src + idx), idx) : E::pad();
        }
    }
    __syncwarp();
    const int bn = xp_addr<LK>(t << LK);
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        v[q] = sm[bn + xp_addr<LK>(q)];
    });
    __syncwarp();
}

// Store the sorted natural-layout tile (lane t holds [t*K, t*K + K)) through
// the shared region so that lane t writes elements t, t + G, ...: coalesced in
// global memory, and conflict-free in shared memory (for register q the G
// lanes read addresses q*G + (q*G >> LK) + t, consecutive banks, and the
// warp's other arrays sit G banks further on).
template <class E, int LK, int LG>
__device__ __forceinline__ void xp_store_striped(typename E::Reg (&v)[1 << LK], typename E::Mem* dst,
                                                 const int t, const int n, typename E::Reg* sm) {
    constexpr int K = 1 << LK, G = 1 << LG;
    const int bn = xp_addr<LK>(t << LK);
    sfor<0, K>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        sm[bn + xp_addr<LK>(q)] = v[q];
    });
    __syncwarp();
    if (n == K * G) {
#pragma unroll
        for (int q = 0; q < K; ++q) xp_stcs(dst + q * G + t, E::to_mem(sm[xp_addr<LK>(q * G + t)]));
    } else {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const int idx = q * G + t;
            const typename E::Reg x = sm[xp_addr<LK>(idx)];
            if (idx < n) xp_stcs(dst + idx, E::to_mem(x));
        }
    }
    __syncwarp();
}

// Packed batch (array a at [a*n, a*n + n)): each warp sorts 32/G arrays at a
// time and strides over the batch by the whole grid.  IO selects how arrays
// move: kXpIoBlocked, each lane its K consecutive elements with 128-bit
// accesses; kXpIoStriped (keys alone), coalesced relabelling loads; kXpIoStaged
// (any element type), coalesced loads through the shared region.  Both
// coalesced forms store through the shared region, coalesced.  PF: the warp loads its next
// arrays into registers before sorting the current ones, so that with a grid
// of a few warps per SM the loads of one round overlap the sorting of the
// previous one.  No CTA-wide barrier: every warp runs on its own.
constexpr int kXpIoBlocked = 0, kXpIoStriped = 1, kXpIoStaged = 2;

template <class E, int LK, int LG, int WPC, int MINB, int IO, bool PF = false>
__global__ void __launch_bounds__(WPC * 32, MINB)
    k_sort_xpose(const typename E::Mem* in, typename E::Mem* out, int n, long long arrays, unsigned opts) {
    constexpr bool STRIPED = IO == kXpIoStriped;
    using R = typename E::Reg;
    constexpr int K = 1 << LK, G = 1 << LG, APW = 32 / G;
    static_assert(LG <= 5 && LG <= LK && LG >= 1, "one warp or less per array, at most two windows");
    static_assert(!STRIPED || !E::kStable, "striped access relabels the input: keys only");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = int(threadIdx.x) >> 5, lane = int(threadIdx.x) & 31;
    const int slot = lane >> LG, t = lane & (G - 1);
    R* sm = reinterpret_cast<R*>(smem_raw) + (warp * APW + slot) * xp_region<LK, LG>();
    const long long stride = (long long)gridDim.x * WPC * APW;
    // Launched with programmatic stream serialization: wait until the
    // preceding kernel of the stream has completed and its writes are
    // visible (immediate without such a predecessor), then let the next
    // launch's CTAs be scheduled as this grid's CTAs retire.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    // With the sortedness check the tile is loaded in its own order (the
    // striped relabelling would hide the input's order from the test).
    const bool check = (opts & kOptSortedCheck) != 0;
    long long first = ((long long)blockIdx.x * WPC + warp) * APW;
    auto load = [&](R (&x)[K], long long a) {
        const int na = a < arrays ? n : 0;
        const typename E::Mem* src = in + (a < arrays ? a : 0) * (long long)n;
        if constexpr (IO == kXpIoStaged) {
            xp_load_staged<E, LK, LG>(x, src, t, na, sm);
        } else {
            if (STRIPED && !check) xp_load_striped<E, LK, LG>(x, src, t, na);
            else load_tile<E, K>(x, src, t * K, na);
        }
    };
    auto finish = [&](R (&x)[K], long long a) {
        bool skip = false;
        if (check) skip = xp_warp_in_order<E, LK, LG>(x, t);
        if (!skip) xp_network<E, LK, LG>(x, t, sm, check);
        if (skip && in == out) return;  // in order and in place: nothing to write
        const int na = a < arrays ? n : 0;
        typename E::Mem* dst = out + (a < arrays ? a : 0) * (long long)n;
        if constexpr (IO != kXpIoBlocked) xp_store_striped<E, LK, LG>(x, dst, t, na, sm);
        else store_tile<E, K>(x, dst, t * K, na);
    };
    R v[K];
    if constexpr (PF) {
        if (first < arrays) load(v, first + slot);
    }
    for (; first < arrays; first += stride) {
        const long long a = first + slot;
        if constexpr (PF) {
            R w[K];
            load(w, a + stride);
            finish(v, a);
#pragma unroll
            for (int q = 0; q < K; ++q) v[q] = w[q];
        } else {
            load(v, a);
            finish(v, a);
        }
    }
}

// The same over a list of CSR arrays (a ragged plan's length class): arrays
// ids[0 .. count) with array a at [off[a], off[a+1]); count and the list's
// first position read on the device when d_count is set; each warp pulls
// its next arrays from the queue at d_head when set (one atomicAdd per
// warp), else strides over the list.
template <class E, int LK, int LG, int MINB, int IO>
__global__ void __launch_bounds__(32, MINB)
    k_sort_xpose_list(const typename E::Mem* in, typename E::Mem* out, const int* __restrict__ off,
                      const int* __restrict__ ids, int count, const int* d_count, const int* d_base, int* d_head) {
    constexpr bool STRIPED = IO == kXpIoStriped;
    using R = typename E::Reg;
    constexpr int K = 1 << LK, G = 1 << LG, APW = 32 / G;
    static_assert(LG <= 5 && LG <= LK && LG >= 1, "one warp or less per array, at most two windows");
    static_assert(!STRIPED || !E::kStable, "striped access relabels the input: keys only");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = int(threadIdx.x) & 31;
    const int slot = lane >> LG, t = lane & (G - 1);
    R* sm = reinterpret_cast<R*>(smem_raw) + slot * xp_region<LK, LG>();
    if (d_count) {
        count = *d_count;
        ids += *d_base;
    }
    long long first = (long long)blockIdx.x * APW;
    for (;;) {
        if (d_head) {
            int f = 0;
            if (lane == 0) f = atomicAdd(d_head, APW);
            first = __shfl_sync(0xffffffffu, f, 0);
        }
        if (first >= count) break;  // uniform across the warp
        const long long g = first + slot;
        int na = 0;
        long long start = 0;
        if (g < count) {
            const int a = ids[g];
            start = off[a];
            na = off[a + 1] - off[a];
        }
        R v[K];
        if constexpr (IO == kXpIoStaged) xp_load_staged<E, LK, LG>(v, in + start, t, na, sm);
        else if constexpr (STRIPED) xp_load_striped<E, LK, LG>(v, in + start, t, na);
        else load_tile<E, K>(v, in + start, t * K, na);
        xp_network<E, LK, LG>(v, t, sm, false);
        if constexpr (IO != kXpIoBlocked) xp_store_striped<E, LK, LG>(v, out + start, t, na, sm);
        else store_tile<E, K>(v, out + start, t * K, na);
        if (!d_head) first += (long long)gridDim.x * APW;
    }
}

}  // namespace b200s
