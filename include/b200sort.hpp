// b200sort.hpp — C++ wrappers over the C ABI with the reference's names.
//
// berenger-eu/cuda-sort exposes its small-array sorts as templates whose
// compile-time arguments pick a kernel configuration (working length,
// threads, and the Sorted / Shared / Async switches), launched by the caller
// one CTA per array over a packed batch (bench.cu:355-393).  The wrappers
// below keep those names and template arguments so that a call site changes
// from a kernel launch to a function call, and run the b200sort kernels:
//
//   reference (launch per batch)                               here
//   Sort_1Block_v6_register<T,W,Th,S,Sh,A><<<A,Th,2W*sizeof(T)>>>(in, out, n)
//     (cusort_v6.hpp:181-184; batched: bench.cu:389-393)      b200sort::Sort_1Block_v6_register<T,W,Th,S,Sh,A>(in, out, n, A)
//   Sort_1Block_v5_static<T,W,Th,S,Sh,A>(in, out, n)           b200sort::Sort_1Block_v5_static<...>(in, out, n, A)
//     (cusort_experiments.hpp:416-419)
//   Sort_1Block_v4_xor<T,S,Sh,A>(in, out, n, working)          b200sort::Sort_1Block_v4_xor<...>(in, out, n, working, A)
//     (cusort_experiments.hpp:411-414)
//   Sort_1Block_gt32_extsm_v3_outofplace<T,S,Sh>(in, out, n, w) b200sort::Sort_1Block_gt32_extsm_v3<...>(in, out, n, w, A)
//     (cusort.hpp:1259-1262)
//   Sort_1Warp_SM_le32_outofplace<T,S,Sh>(in, out, n)          b200sort::Sort_1Warp_SM_le32<...>(in, out, n, A)
//     (cusort.hpp:603-606)
//
// Template arguments are checked as the reference checks them (static_assert
// where it static_asserts, a status where it asserts on the device), but the
// kernel configuration is chosen by b200sort's tile table: every variant
// produces the reference's exact output, including the order of records with
// equal keys.  Element types: int, uint64_t, and any 8-byte record laid out
// as {int key; int payload;} such as the reference's IntAndData
// (intanddata.hpp:9-11), or a 16-byte {uint64_t key; int payload; int pad;}.
#ifndef B200SORT_HPP
#define B200SORT_HPP

#include <cstdint>
#include <type_traits>

#include "b200sort.h"

namespace b200sort {

template <class T, class = void>
struct dtype_of {
    // 8-byte records {int key; int payload;} (IntAndData) and 16-byte
    // {uint64_t key; int payload; int pad;} records.
    static_assert(std::is_trivially_copyable<T>::value && (sizeof(T) == 8 || sizeof(T) == 16),
                  "b200sort sorts int, uint64_t, {int,int} and {uint64_t,int,int} elements");
    static constexpr b200s_dtype value = sizeof(T) == 8 ? B200S_I32_I32 : B200S_U64_I32;
};
template <>
struct dtype_of<int> {
    static constexpr b200s_dtype value = B200S_I32;
};
template <>
struct dtype_of<std::uint64_t> {
    static constexpr b200s_dtype value = B200S_U64;
};

// Sort `arrays` packed arrays (array a at input + a*n) into output (may equal
// input).  The generic entry every named wrapper forwards to.
template <class T>
inline b200s_status sort_packed(const T* input, T* output, int n, long long arrays = 1, unsigned flags = 0,
                                void* stream = nullptr) {
    return b200s_sort_packed(dtype_of<T>::value, input, output, n, arrays, flags, nullptr, stream);
}

constexpr bool is_pow2(unsigned x) { return x && !(x & (x - 1)); }

// cusort_v6.hpp:130-147: Working a power of two >= 32, Threads a power of two
// in [32, min(1024, Working)], at most 16 values per thread, 0 < n <= Working.
template <typename T, unsigned Working, unsigned Threads, bool Sorted, bool Shared, bool Async>
inline b200s_status Sort_1Block_v6_register(T* input, T* output, int validCount, long long arrays = 1,
                                            void* stream = nullptr) {
    static_assert(Working >= 32 && is_pow2(Working), "Power-of-two working length required");
    static_assert(Threads >= 32 && Threads <= 1024 && Threads <= Working && is_pow2(Threads),
                  "Power-of-two block size required");
    static_assert(Working / Threads <= 16, "v6 limits register tiles to 16 values per thread");
    if (validCount <= 0 || unsigned(validCount) > Working) return B200S_ERR_INVALID_ARGUMENT;
    return sort_packed(input, output, validCount, arrays, Sorted ? B200S_SORTED_CHECK : 0u, stream);
}

// cusort_experiments.hpp:366-419 (V5: static sizes; V4: runtime working length).
template <typename T, unsigned WorkingValues, unsigned BlockThreads, bool TestIfSorted, bool FullSM,
          bool AsyncCopy>
inline b200s_status Sort_1Block_v5_static(T* input, T* output, int n, long long arrays = 1,
                                          void* stream = nullptr) {
    static_assert(WorkingValues >= 32 && is_pow2(WorkingValues), "Power-of-two working length required");
    static_assert(BlockThreads >= 32 && BlockThreads <= 1024 && is_pow2(BlockThreads) &&
                      BlockThreads <= WorkingValues,
                  "Power-of-two block size required");
    if (n <= 0 || unsigned(n) > WorkingValues) return B200S_ERR_INVALID_ARGUMENT;
    return sort_packed(input, output, n, arrays, TestIfSorted ? B200S_SORTED_CHECK : 0u, stream);
}

template <typename T, bool TestIfSorted, bool FullSM, bool AsyncCopy>
inline b200s_status Sort_1Block_v4_xor(T* input, T* output, int n, unsigned working, long long arrays = 1,
                                       void* stream = nullptr) {
    if (n <= 0 || working < 32 || !is_pow2(working) || unsigned(n) > working) return B200S_ERR_INVALID_ARGUMENT;
    return sort_packed(input, output, n, arrays, TestIfSorted ? B200S_SORTED_CHECK : 0u, stream);
}

// cusort.hpp:1229-1262 (V3, out of place) and cusort.hpp:574-606 (warp, n <= 32).
template <typename T, bool TestIfSorted, bool FullSM>
inline b200s_status Sort_1Block_gt32_extsm_v3(T* input, T* output, int n, int working, long long arrays = 1,
                                              void* stream = nullptr) {
    if (n <= 0 || working < n || !is_pow2(unsigned(working))) return B200S_ERR_INVALID_ARGUMENT;
    return sort_packed(input, output, n, arrays, TestIfSorted ? B200S_SORTED_CHECK : 0u, stream);
}

template <typename T, bool TestIfSorted, bool FullSM>
inline b200s_status Sort_1Warp_SM_le32(T* input, T* output, int n, long long arrays = 1, void* stream = nullptr) {
    if (n <= 0 || n > 32) return B200S_ERR_INVALID_ARGUMENT;
    return sort_packed(input, output, n, arrays, TestIfSorted ? B200S_SORTED_CHECK : 0u, stream);
}

// Ragged batches (the reference's partition sort over CSR ranges,
// SortPartitionsAdaptive_outofplace, cusort.hpp:2309-2352) through a plan.
class Plan {
public:
    template <class T>
    static Plan create(long long max_arrays, unsigned flags = 0, int device = 0) {
        Plan p;
        p.status_ = b200s_plan_create(&p.plan_, dtype_of<T>::value, flags, max_arrays, device);
        return p;
    }
    Plan() = default;
    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;
    Plan(Plan&& o) noexcept : plan_(o.plan_), status_(o.status_) { o.plan_ = nullptr; }
    ~Plan() {
        if (plan_) b200s_plan_destroy(plan_);
    }
    b200s_status status() const { return status_; }
    template <class T>
    b200s_status sort(const T* input, T* output, const int* d_offsets, long long arrays, void* stream = nullptr) {
        return b200s_sort_ragged(plan_, input, output, d_offsets, arrays, stream);
    }

private:
    b200s_plan* plan_ = nullptr;
    b200s_status status_ = B200S_ERR_INVALID_ARGUMENT;
};

// The leaf of the partitioned large-array sort, under the reference kernel's
// name (cusort.hpp:2309-2352): a host call that replaces the launch
//   SortPartitionsAdaptive_outofplace<T, TestIfSorted, FullSM>
//       <<<nbParts, threads, shared, stream>>>(input, output, counterParts, uniformParts, nbParts);
// (cusort.hpp:2624-2627) with the same arguments; see b200s_sort_partitions.
template <typename T, bool TestIfSorted = false, bool FullSM = false>
inline b200s_status SortPartitionsAdaptive_outofplace(const T* input, T* output, const int* counterParts,
                                                      const int* uniformParts, int nbParts,
                                                      void* stream = nullptr) {
    return b200s_sort_partitions(dtype_of<T>::value, TestIfSorted ? B200S_SORTED_CHECK : 0u, input, output,
                                 counterParts, uniformParts, nbParts, stream);
}

}  // namespace b200sort

#endif  // B200SORT_HPP
