// Element types and their comparison rules for the batched bitonic sort.
//
// Memory layouts (what the caller's buffers hold):
//   int32_t   keys only                                   4 B
//   RecI32    {int32 key; int32 data;}  == IntAndData     8 B  (intanddata.hpp:9-11)
//   uint64_t  keys only                                   8 B
//   RecU64    {uint64 key; int32 data; int32 reserved;}  16 B  (AoS; reserved is written as 0)
//
// Register forms (what a thread holds while sorting) add an original-position
// word in the stable mode, so that ties are broken by input order.
//
// Ordering follows the reference: records compare by key only
// (intanddata.hpp:20-31) and, on the default path, a comparator keeps its own
// element on ties: min(a,b) = b<a ? b : a, max(a,b) = a<b ? b : a
// (cusort.hpp:460-472).  Padding uses the maximum key with a maximum payload
// (cusort.hpp:257-271, intanddata.hpp:47-52).
#pragma once
#include <climits>
#include <cstdint>

namespace b200s {

struct RecI32 {
    int32_t key;
    int32_t data;
};
struct __align__(16) RecU64 {
    uint64_t key;
    int32_t data;
    int32_t reserved;
};

// Element J of a 16-byte word, and the inverse, for each memory layout; J is
// a compile-time index so the moves stay in registers.
template <int J>
__device__ __forceinline__ void from_u4(const uint4& u, int32_t& m) {
    m = int32_t(J == 0 ? u.x : J == 1 ? u.y : J == 2 ? u.z : u.w);
}
template <int J>
__device__ __forceinline__ void to_u4(uint4& u, int32_t m) {
    if constexpr (J == 0) u.x = uint32_t(m);
    else if constexpr (J == 1) u.y = uint32_t(m);
    else if constexpr (J == 2) u.z = uint32_t(m);
    else u.w = uint32_t(m);
}
template <int J>
__device__ __forceinline__ void from_u4(const uint4& u, uint64_t& m) {
    m = J == 0 ? (uint64_t(u.y) << 32 | u.x) : (uint64_t(u.w) << 32 | u.z);
}
template <int J>
__device__ __forceinline__ void to_u4(uint4& u, uint64_t m) {
    if constexpr (J == 0) {
        u.x = uint32_t(m);
        u.y = uint32_t(m >> 32);
    } else {
        u.z = uint32_t(m);
        u.w = uint32_t(m >> 32);
    }
}
template <int J>
__device__ __forceinline__ void from_u4(const uint4& u, RecI32& m) {
    m.key = int32_t(J == 0 ? u.x : u.z);
    m.data = int32_t(J == 0 ? u.y : u.w);
}
template <int J>
__device__ __forceinline__ void to_u4(uint4& u, const RecI32& m) {
    if constexpr (J == 0) {
        u.x = uint32_t(m.key);
        u.y = uint32_t(m.data);
    } else {
        u.z = uint32_t(m.key);
        u.w = uint32_t(m.data);
    }
}
template <int J>
__device__ __forceinline__ void from_u4(const uint4& u, RecU64& m) {
    m.key = uint64_t(u.y) << 32 | u.x;
    m.data = int32_t(u.z);
    m.reserved = int32_t(u.w);
}
template <int J>
__device__ __forceinline__ void to_u4(uint4& u, const RecU64& m) {
    u.x = uint32_t(m.key);
    u.y = uint32_t(m.key >> 32);
    u.z = uint32_t(m.data);
    u.w = uint32_t(m.reserved);
}

__device__ __forceinline__ uint32_t shfl_x(uint32_t v, int m) {
    return __shfl_xor_sync(0xffffffffu, v, m);
}
__device__ __forceinline__ int32_t shfl_x(int32_t v, int m) {
    return __shfl_xor_sync(0xffffffffu, v, m);
}
__device__ __forceinline__ uint64_t shfl_x(uint64_t v, int m) {
    return __shfl_xor_sync(0xffffffffu, (unsigned long long)v, m);
}
__device__ __forceinline__ int32_t shfl_d(int32_t v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
__device__ __forceinline__ uint64_t shfl_d(uint64_t v, int d) {
    return __shfl_down_sync(0xffffffffu, (unsigned long long)v, d);
}

// ---- int32 keys --------------------------------------------------------------
struct ElemI32 {
    static constexpr bool kKeysOnly = true;  // tie order unobservable
    using Mem = int32_t;
    using Reg = int32_t;
    static constexpr bool kStable = false;
    static constexpr bool kCompact = false;
    static __device__ __forceinline__ Reg pad() { return INT32_MAX; }
    static __device__ __forceinline__ Reg from_mem(Mem m, int) { return m; }
    static __device__ __forceinline__ Mem to_mem(Reg r) { return r; }
    static __device__ __forceinline__ Reg shfl(Reg v, int m) { return shfl_x(v, m); }
    static __device__ __forceinline__ Reg shfl_down(Reg v, int d) { return shfl_d(v, d); }
    // b belongs before a (the pair (a, b) is out of order).
    static __device__ __forceinline__ bool after(Reg a, Reg b) { return b < a; }
    // Ascending compare-exchange of (lower, upper).  Equal keys are
    // indistinguishable, so min/max is the keep-own rule.
    static __device__ __forceinline__ void cex(Reg& lo, Reg& hi) {
        const Reg a = lo, b = hi;
        lo = min(a, b);
        hi = max(a, b);
    }
    // One side of a cross-thread compare-exchange: the upper side keeps the
    // larger, the lower side the smaller.
    static __device__ __forceinline__ Reg pick(Reg own, Reg other, bool upper) {
        return upper ? max(own, other) : min(own, other);
    }
};

// int32 keys through the compact network: for the 4- and 8-CTA cluster tiles,
// whose fully unrolled network spills at 128 registers (432-728 bytes); the
// compact form does not, and is 5-8 % faster there (16 M keys, n = 65536:
// 0.43 -> 0.40 ms; 131072: 0.61 -> 0.58 ms).  Same comparators, same output.
struct ElemI32C : ElemI32 {
    static constexpr bool kCompact = true;
};

// ---- uint64 keys -------------------------------------------------------------
struct ElemU64 {
    static constexpr bool kKeysOnly = true;
    using Mem = uint64_t;
    using Reg = uint64_t;
    static constexpr bool kStable = false;
    static constexpr bool kCompact = true;
    static __device__ __forceinline__ Reg pad() { return UINT64_MAX; }
    static __device__ __forceinline__ Reg from_mem(Mem m, int) { return m; }
    static __device__ __forceinline__ Mem to_mem(Reg r) { return r; }
    static __device__ __forceinline__ Reg shfl(Reg v, int m) { return shfl_x(v, m); }
    static __device__ __forceinline__ Reg shfl_down(Reg v, int d) { return shfl_d(v, d); }
    static __device__ __forceinline__ bool after(Reg a, Reg b) { return b < a; }
    static __device__ __forceinline__ void cex(Reg& lo, Reg& hi) {
        const Reg a = lo, b = hi;
        const bool sw = b < a;
        lo = sw ? b : a;
        hi = sw ? a : b;
    }
    static __device__ __forceinline__ Reg pick(Reg own, Reg other, bool upper) {
        const bool take = upper ? (own < other) : (other < own);
        return take ? other : own;
    }
};

// ---- records: int32 key + int32 payload (IntAndData) ------------------------
struct RegRecI32 {
    int32_t key;
    int32_t data;
};
struct ElemRecI32 {
    using Mem = RecI32;
    using Reg = RegRecI32;
    static constexpr bool kStable = false;
    static constexpr bool kCompact = true;
    static __device__ __forceinline__ Reg pad() { return Reg{INT32_MAX, INT32_MAX}; }
    static __device__ __forceinline__ Reg from_mem(Mem m, int) { return Reg{m.key, m.data}; }
    static __device__ __forceinline__ Mem to_mem(Reg r) { return Mem{r.key, r.data}; }
    static __device__ __forceinline__ Reg shfl(Reg v, int m) {
        return Reg{shfl_x(v.key, m), shfl_x(v.data, m)};
    }
    static __device__ __forceinline__ Reg shfl_down(Reg v, int d) { return Reg{shfl_d(v.key, d), shfl_d(v.data, d)}; }
    static __device__ __forceinline__ bool after(const Reg& a, const Reg& b) { return b.key < a.key; }
    static __device__ __forceinline__ void cex(Reg& lo, Reg& hi) {
        const Reg a = lo, b = hi;
        const bool sw = b.key < a.key;          // strict: ties keep their places
        lo.key = sw ? b.key : a.key;
        lo.data = sw ? b.data : a.data;
        hi.key = sw ? a.key : b.key;
        hi.data = sw ? a.data : b.data;
    }
    static __device__ __forceinline__ Reg pick(Reg own, Reg other, bool upper) {
        const bool take = upper ? (own.key < other.key) : (other.key < own.key);
        return Reg{take ? other.key : own.key, take ? other.data : own.data};
    }
};

// Stable mode for IntAndData: (key, original position) is unique, so the
// network output equals a stable sort by key.
struct RegRecI32S {
    int32_t key;
    int32_t data;
    int32_t pos;
};
struct ElemRecI32S {
    using Mem = RecI32;
    using Reg = RegRecI32S;
    static constexpr bool kStable = true;
    static constexpr bool kCompact = true;
    static __device__ __forceinline__ Reg pad() { return Reg{INT32_MAX, INT32_MAX, INT32_MAX}; }
    static __device__ __forceinline__ Reg from_mem(Mem m, int pos) { return Reg{m.key, m.data, pos}; }
    static __device__ __forceinline__ Mem to_mem(Reg r) { return Mem{r.key, r.data}; }
    static __device__ __forceinline__ Reg shfl(Reg v, int m) {
        return Reg{shfl_x(v.key, m), shfl_x(v.data, m), shfl_x(v.pos, m)};
    }
    static __device__ __forceinline__ Reg shfl_down(Reg v, int d) {
        return Reg{shfl_d(v.key, d), shfl_d(v.data, d), shfl_d(v.pos, d)};
    }
    static __device__ __forceinline__ bool lt(const Reg& a, const Reg& b) {
        return a.key < b.key || (a.key == b.key && a.pos < b.pos);
    }
    static __device__ __forceinline__ bool after(const Reg& a, const Reg& b) { return lt(b, a); }
    static __device__ __forceinline__ void cex(Reg& lo, Reg& hi) {
        const Reg a = lo, b = hi;
        const bool sw = lt(b, a);
        lo.key = sw ? b.key : a.key;
        lo.data = sw ? b.data : a.data;
        lo.pos = sw ? b.pos : a.pos;
        hi.key = sw ? a.key : b.key;
        hi.data = sw ? a.data : b.data;
        hi.pos = sw ? a.pos : b.pos;
    }
    static __device__ __forceinline__ Reg pick(Reg own, Reg other, bool upper) {
        const bool take = upper ? lt(own, other) : lt(other, own);
        Reg r;
        r.key = take ? other.key : own.key;
        r.data = take ? other.data : own.data;
        r.pos = take ? other.pos : own.pos;
        return r;
    }
};

// ---- records: uint64 key + int32 payload -------------------------------------
struct alignas(16) RegRecU64 {
    uint64_t key;
    int32_t data;
};
struct ElemRecU64 {
    using Mem = RecU64;
    using Reg = RegRecU64;
    static constexpr bool kStable = false;
    static constexpr bool kCompact = true;
    static __device__ __forceinline__ Reg pad() { return Reg{UINT64_MAX, INT32_MAX}; }
    static __device__ __forceinline__ Reg from_mem(Mem m, int) { return Reg{m.key, m.data}; }
    static __device__ __forceinline__ Mem to_mem(Reg r) { return Mem{r.key, r.data, 0}; }
    static __device__ __forceinline__ Reg shfl(Reg v, int m) {
        return Reg{shfl_x(v.key, m), shfl_x(v.data, m)};
    }
    static __device__ __forceinline__ Reg shfl_down(Reg v, int d) { return Reg{shfl_d(v.key, d), shfl_d(v.data, d)}; }
    static __device__ __forceinline__ bool after(const Reg& a, const Reg& b) { return b.key < a.key; }
    // Field by field: whole-struct selects of this padded register record
    // made the compiler spill in the large tiles.
    static __device__ __forceinline__ void cex(Reg& lo, Reg& hi) {
        const Reg a = lo, b = hi;
        const bool sw = b.key < a.key;
        lo.key = sw ? b.key : a.key;
        lo.data = sw ? b.data : a.data;
        hi.key = sw ? a.key : b.key;
        hi.data = sw ? a.data : b.data;
    }
    static __device__ __forceinline__ Reg pick(Reg own, Reg other, bool upper) {
        const bool take = upper ? (own.key < other.key) : (other.key < own.key);
        Reg r;
        r.key = take ? other.key : own.key;
        r.data = take ? other.data : own.data;
        return r;
    }
};

struct alignas(16) RegRecU64S {
    uint64_t key;
    int32_t data;
    int32_t pos;
};
struct ElemRecU64S {
    using Mem = RecU64;
    using Reg = RegRecU64S;
    static constexpr bool kStable = true;
    static constexpr bool kCompact = true;
    static __device__ __forceinline__ Reg pad() { return Reg{UINT64_MAX, INT32_MAX, INT32_MAX}; }
    static __device__ __forceinline__ Reg from_mem(Mem m, int pos) { return Reg{m.key, m.data, pos}; }
    static __device__ __forceinline__ Mem to_mem(Reg r) { return Mem{r.key, r.data, 0}; }
    static __device__ __forceinline__ Reg shfl(Reg v, int m) {
        return Reg{shfl_x(v.key, m), shfl_x(v.data, m), shfl_x(v.pos, m)};
    }
    static __device__ __forceinline__ Reg shfl_down(Reg v, int d) {
        return Reg{shfl_d(v.key, d), shfl_d(v.data, d), shfl_d(v.pos, d)};
    }
    static __device__ __forceinline__ bool lt(const Reg& a, const Reg& b) {
        return a.key < b.key || (a.key == b.key && a.pos < b.pos);
    }
    static __device__ __forceinline__ bool after(const Reg& a, const Reg& b) { return lt(b, a); }
    static __device__ __forceinline__ void cex(Reg& lo, Reg& hi) {
        const Reg a = lo, b = hi;
        const bool sw = lt(b, a);
        lo.key = sw ? b.key : a.key;
        lo.data = sw ? b.data : a.data;
        lo.pos = sw ? b.pos : a.pos;
        hi.key = sw ? a.key : b.key;
        hi.data = sw ? a.data : b.data;
        hi.pos = sw ? a.pos : b.pos;
    }
    static __device__ __forceinline__ Reg pick(Reg own, Reg other, bool upper) {
        const bool take = upper ? lt(own, other) : lt(other, own);
        Reg r;
        r.key = take ? other.key : own.key;
        r.data = take ? other.data : own.data;
        r.pos = take ? other.pos : own.pos;
        return r;
    }
};

// uint64 keys alone are totally ordered values: the stable mode changes nothing.

// Shared-memory (and distributed-shared-memory) element accesses.  The
// 16-byte register records move as one 128-bit access: field by field (an
// 8-byte key, then a 4-byte payload at a 16-byte stride) each access takes
// two wavefronts per half-warp instead of one per quarter-warp.
template <class R>
__device__ __forceinline__ R sh_ld(const R* p) {
    return *p;
}
template <class R>
__device__ __forceinline__ void sh_st(R* p, const R& v) {
    *p = v;
}
// The fourth word is padding: one 128-bit shared-space load in PTX (p is in
// this CTA's shared memory), so that the compiler does not narrow it to an
// 8-byte and a 4-byte load.
__device__ __forceinline__ RegRecU64 sh_ld(const RegRecU64* p) {
    unsigned x, y, z, w;
    const unsigned a = unsigned(__cvta_generic_to_shared(p));
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(x), "=r"(y), "=r"(z), "=r"(w) : "r"(a) : "memory");
    (void)w;
    return RegRecU64{(uint64_t(y) << 32) | x, int32_t(z)};
}
__device__ __forceinline__ void sh_st(RegRecU64* p, const RegRecU64& v) {
    *reinterpret_cast<uint4*>(p) = make_uint4(unsigned(v.key), unsigned(v.key >> 32), unsigned(v.data), 0u);
}
// Reads of a cluster peer's shared memory (a generic pointer from
// map_shared_rank): plain loads, 128 bits for the 16-byte records.
template <class R>
__device__ __forceinline__ R dsm_ld(const R* p) {
    return *p;
}
__device__ __forceinline__ RegRecU64 dsm_ld(const RegRecU64* p) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    return RegRecU64{(uint64_t(u.y) << 32) | u.x, int32_t(u.z)};
}
__device__ __forceinline__ RegRecU64S dsm_ld(const RegRecU64S* p) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    return RegRecU64S{(uint64_t(u.y) << 32) | u.x, int32_t(u.z), int32_t(u.w)};
}
__device__ __forceinline__ RegRecU64S sh_ld(const RegRecU64S* p) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    return RegRecU64S{(uint64_t(u.y) << 32) | u.x, int32_t(u.z), int32_t(u.w)};
}
__device__ __forceinline__ void sh_st(RegRecU64S* p, const RegRecU64S& v) {
    *reinterpret_cast<uint4*>(p) =
        make_uint4(unsigned(v.key), unsigned(v.key >> 32), unsigned(v.data), unsigned(v.pos));
}

}  // namespace b200s
