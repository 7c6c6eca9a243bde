// b200s_sort_ragged_noalloc: the ragged sort for callers that cannot
// allocate device memory.
//
// Some callers of a sorting library cannot call cudaMalloc: plugins living
// inside a host framework that already owns all device memory through its
// own pool (a second allocator would fail or fragment that pool), and
// latency-critical loops where cudaMalloc's implicit device-wide
// synchronisation would stall unrelated work.  For them this entry point runs
// the same kernels as b200s_sort_ragged, but keeps the scratch those kernels
// need (the bucket counters and the array-id lists) in one file-scope
// __device__ array instead of a plan's allocation.
//
// The array is sized for B200S_NOALLOC_MAX_ARRAYS arrays (about 640 KiB) and
// every GPU that loads this library holds it until the process exits.  In
// host code its name stands for a host-side shadow, not for device memory, so
// the kernels receive the device address from cudaGetSymbolAddress, looked up
// once per device on that device's first call.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "b200sort.h"
#include "ragged.cuh"
#include "registry.h"

namespace b200s {

b200s_status set_error(b200s_status s, const std::string& msg);
b200s_status cuda_error(cudaError_t e, const char* what);
int effective_stable(int dtype, uint32_t flags);
unsigned ragged_family_mask(int dtype, int stable);
unsigned ragged_dedicated_mask(int dtype, int stable);
void dedicated_entries(int dtype, int stable, int nb, unsigned* mask, int* idx, bool* xc);
bool cluster_xc(int dtype, int stable, int entry);
int lookup_default_entry(int dtype, int stable, long long n, int* persistent);

namespace {

constexpr int kNoAllocArrays = B200S_NOALLOC_MAX_ARRAYS;

struct NoAllocScratch {
    RaggedCtl ctl;
    int ids[kNoAllocArrays];
    int oids[kMaxOverflow * kNoAllocArrays];
};

}  // namespace

// The scratch itself: control block, bucketed ids, cluster-bucket ids.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.
b200s_status scratch_address(NoAllocScratch** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error(B200S_ERR_UNSUPPORTED, "device index beyond 63");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_ptr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_scratch_ptr[dev];
    return B200S_OK;
}

const RaggedEntry* ragged_entry(int dtype, int stable) {
    for (const RaggedEntry& e : ragged_registry())
        if (e.dtype == dtype && e.stable == stable) return &e;
    return nullptr;
}

}  // namespace
}  // namespace b200s

using namespace b200s;

extern "C" b200s_status b200s_sort_ragged_noalloc(b200s_dtype dtype, uint32_t flags, const void* d_in,
                                                  void* d_out, const int32_t* d_offsets, int64_t arrays,
                                                  void* stream) {
    if (dtype < 0 || dtype > 3) return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (flags & ~(B200S_STABLE | B200S_SORTED_CHECK))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown flag bits");
    if (arrays < 0) return set_error(B200S_ERR_INVALID_ARGUMENT, "negative array count");
    if (arrays > kNoAllocArrays)
        return set_error(B200S_ERR_INVALID_ARGUMENT,
                         "b200s_sort_ragged_noalloc: " + std::to_string(arrays) +
                             " arrays exceed the fixed scratch of B200S_NOALLOC_MAX_ARRAYS = " +
                             std::to_string(kNoAllocArrays) + " (use a plan for larger batches)");
    if (arrays == 0) return B200S_OK;
    if (!d_in || !d_out || !d_offsets) return set_error(B200S_ERR_INVALID_ARGUMENT, "null buffer");
    const int stable = effective_stable(dtype, flags);
    const RaggedEntry* rk = ragged_entry(dtype, stable);
    if (!rk) return set_error(B200S_ERR_UNSUPPORTED, "no ragged kernel for this dtype");
    NoAllocScratch* s = nullptr;
    b200s_status st = scratch_address(&s);
    if (st != B200S_OK) return st;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_error(e, "device attributes");
    const int per_sm = rk->resident_per_sm();
    if (per_sm <= 0) return set_error(B200S_ERR_CUDA, "ragged kernel does not fit on this device");

    BinSpec spec;
    int cluster_idx[kMaxOverflow] = {};
    spec.nb = rk->nb;
    spec.over_lo = kRaggedLmin + rk->nb;
    spec.n_over = overflow_entries(dtype, stable, spec.over_lo, cluster_idx);
    spec.stride = kNoAllocArrays;

    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    const int n = int(arrays);
    // The counters are shared with every other call: start them at zero.
    e = cudaMemsetAsync(&s->ctl, 0, sizeof(RaggedCtl), cs);
    if (e != cudaSuccess) return cuda_error(e, "scratch reset");
    const int bin_threads = 256;
    const int bin_grid = std::max(1, std::min(sms * 4, (n + bin_threads - 1) / bin_threads));
    k_bin_count<<<bin_grid, bin_threads, 0, cs>>>(d_offsets, n, &s->ctl, spec);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "bin count launch");
    k_bin_scatter<<<bin_grid, bin_threads, 0, cs>>>(d_offsets, n, &s->ctl, s->ids, s->oids, spec);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "bin scatter launch");
    // the plan's routing: buckets with their own launch run after the
    // persistent kernel on the same stream (no side streams here); the tile
    // table that sets it loads on the first lookup
    int unused_form = 0;
    (void)lookup_default_entry(dtype, stable, 1, &unused_form);
    unsigned dedicated = ragged_dedicated_mask(dtype, stable);
    int dedicated_idx[kMaxBuckets] = {};
    bool dedicated_xc[kMaxBuckets] = {};
    dedicated_entries(dtype, stable, rk->nb, &dedicated, dedicated_idx, dedicated_xc);
    if (dedicated != (1u << rk->nb) - 1u) {
        e = rk->launch(d_in, d_out, d_offsets, s->ids, &s->ctl, ragged_family_mask(dtype, stable), dedicated,
                       sms * per_sm, cs);
        if (e != cudaSuccess) return cuda_error(e, "ragged sort launch");
    }
    for (int b = rk->nb - 1; b >= 0; --b) {
        if (!((dedicated >> b) & 1u)) continue;
        const KernelEntry& k = registry()[size_t(dedicated_idx[b])];
        e = (dedicated_xc[b] ? k.launch_list_dev_xc : k.launch_list_dev)(
            d_in, d_out, d_offsets, s->ids, &s->ctl.count[b], &s->ctl.base[b], &s->ctl.dhead[b], n, cs);
        if (e != cudaSuccess) return cuda_error(e, "dedicated bucket launch");
    }
    for (int i = 0; i < spec.n_over; ++i) {
        const KernelEntry& k = registry()[size_t(cluster_idx[i])];
        e = (cluster_xc(dtype, stable, cluster_idx[i]) ? k.launch_cluster_list_xc : k.launch_cluster_list)(
            d_in, d_out, d_offsets, s->oids + size_t(i) * kNoAllocArrays, &s->ctl.ocount[i], n, cs);
        if (e != cudaSuccess) return cuda_error(e, "cluster bucket launch");
    }
    return B200S_OK;
}
