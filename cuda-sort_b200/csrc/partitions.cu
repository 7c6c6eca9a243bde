// b200s_sort_partitions: the leaf of the reference's large-array sort.
//
// The reference's partitioned sort (HybridSortPartitionedV3, cusort.hpp:2493-
// 2653) splits one large array into up to 1024 key-range partitions (CSR
// counters), then sorts every small partition in one launch of
// SortPartitionsAdaptive_outofplace (cusort.hpp:2309-2352, launched at
// cusort.hpp:2616-2628) and each larger one with a merge sort.  This entry
// point has that kernel's contract -- values, CSR counters, per-partition
// single-value flags, partition count, out of place -- and runs the ragged
// launch (b200s_sort_ragged) over the partitions, so a partitioned sort that
// calls it inherits the persistent bucketed kernels, including partitions up
// to b200s_ragged_max_length that the reference sends to its merge path.
//
// The ragged launch needs a plan (bucket counters, id lists, a captured
// graph).  Plans are cached per (device, element type, stable, stream) and
// grown to the largest partition count seen; b200s_release_partition_plans
// frees them.  Calls on one stream are ordered by the stream; calls on
// different streams use different plans.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "b200sort.h"

namespace b200s {
b200s_status set_error(b200s_status s, const std::string& msg);
b200s_status cuda_error(cudaError_t e, const char* what);
int effective_stable(int dtype, uint32_t flags);
}  // namespace b200s

using namespace b200s;

namespace {

struct CachedPlan {
    b200s_plan* plan = nullptr;
    int64_t capacity = 0;
};
using PlanKey = std::tuple<int, int, int, void*>;  // device, dtype, stable, stream
std::mutex g_plan_mutex;
std::map<PlanKey, CachedPlan>& plan_cache() {
    static std::map<PlanKey, CachedPlan> cache;
    return cache;
}

}  // namespace

extern "C" {

b200s_status b200s_sort_partitions(b200s_dtype dtype, uint32_t flags, const void* d_in, void* d_out,
                                   const int32_t* d_counters, const int32_t* d_uniform, int32_t nb_parts,
                                   void* stream) {
    (void)d_uniform;  // a single-valued partition sorts to itself: sorting it is the copy
    if (dtype < 0 || dtype > 3) return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (flags & ~(B200S_STABLE | B200S_SORTED_CHECK))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown flag bits");
    if (nb_parts < 0) return set_error(B200S_ERR_INVALID_ARGUMENT, "negative partition count");
    if (nb_parts == 0) return B200S_OK;
    if (!d_in || !d_out || !d_counters) return set_error(B200S_ERR_INVALID_ARGUMENT, "null buffer");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    const int stable = effective_stable(dtype, flags);
    b200s_plan* plan = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_plan_mutex);
        CachedPlan& c = plan_cache()[PlanKey(dev, int(dtype), stable, stream)];
        if (c.capacity < nb_parts) {
            if (c.plan) b200s_plan_destroy(c.plan);
            c.plan = nullptr;
            c.capacity = 0;
            int64_t cap = 1024;  // the reference's partition count limit (MaxNbParts)
            while (cap < nb_parts) cap *= 2;
            const b200s_status st = b200s_plan_create(&c.plan, dtype, stable ? B200S_STABLE : 0u, cap, dev);
            if (st != B200S_OK) return st;
            c.capacity = cap;
        }
        plan = c.plan;
    }
    return b200s_sort_ragged(plan, d_in, d_out, d_counters, nb_parts, stream);
}

b200s_status b200s_release_partition_plans(void) {
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    for (auto& kv : plan_cache())
        if (kv.second.plan) b200s_plan_destroy(kv.second.plan);
    plan_cache().clear();
    return B200S_OK;
}

}  // extern "C"
