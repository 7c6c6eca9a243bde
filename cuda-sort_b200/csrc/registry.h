// Host-side registry of compiled sort kernels (one entry per tile shape and
// element type).  Each translation unit that instantiates kernels appends its
// entries; the C ABI picks one by (dtype, stable, working length).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "opts.h"

namespace b200s {

// opts: launch options (kOptSortedCheck in network.cuh; cluster kernels ignore them).
using PackedLaunch = cudaError_t (*)(const void* in, void* out, int n, long long arrays,
                                     long long grid, cudaStream_t stream, unsigned opts);
using AttrQuery = cudaError_t (*)(cudaFuncAttributes* attr);
// Launch over a list of array ids of a CSR batch (plain per-length launches).
using ListLaunch = cudaError_t (*)(const void* in, void* out, const int* d_off, const int* d_ids,
                                   int count, cudaStream_t stream);
// The same with the count and the list's first position read on the device
// (a dedicated bucket of a ragged plan): at most max_count arrays.
using ListLaunchDev = cudaError_t (*)(const void* in, void* out, const int* d_off, const int* d_ids,
                                      const int* d_count, const int* d_base, int* d_head, int max_count,
                                      cudaStream_t stream);

struct KernelEntry {
    int dtype;        // b200s_dtype
    int stable;       // 0/1
    int lk, lg, lw;   // tile shape
    int cta;          // threads per CTA
    int log2w;        // working length exponent
    size_t smem;      // dynamic shared memory bytes
    int apc;          // arrays per CTA
    PackedLaunch launch;      // one group per array, grid covers the batch
    AttrQuery attrs;
    ListLaunch launch_list;
    PackedLaunch launch_pf;   // persistent grid, next-array prefetch
    int lc;                   // log2 CTAs per array (cluster kernels); -1 for single-CTA tiles
    // Cluster kernels only: sort the arrays ids[0 .. *d_count) of a CSR batch,
    // with the count read on the device (at most max_count).
    cudaError_t (*launch_cluster_list)(const void* in, void* out, const int* d_off, const int* d_ids,
                                       const int* d_count, int max_count, cudaStream_t stream);
    ListLaunchDev launch_list_dev;  // single-CTA tiles only (null for cluster kernels)
    // Launch form 3 of a multi-warp or cluster tile: the same tile running the
    // transposed network of cta_xpose.cuh (null where none is compiled).
    // Packed batch, host-counted id list, device-counted id list (single-CTA
    // tiles) and cluster id list with a device count (cluster tiles).
    PackedLaunch launch_xc = nullptr;
    ListLaunch launch_list_xc = nullptr;
    ListLaunchDev launch_list_dev_xc = nullptr;
    cudaError_t (*launch_cluster_list_xc)(const void* in, void* out, const int* d_off, const int* d_ids,
                                          const int* d_count, int max_count, cudaStream_t stream) = nullptr;
    size_t smem_xc = 0;  // its dynamic shared memory bytes
};

void register_i32(std::vector<KernelEntry>& out);
void register_i32_alt(std::vector<KernelEntry>& out);  // called by register_i32
void register_rec(std::vector<KernelEntry>& out);
void register_u64(std::vector<KernelEntry>& out);
void register_cluster_keys(std::vector<KernelEntry>& out);
void register_cluster_rec(std::vector<KernelEntry>& out);
void register_cluster_u64rec(std::vector<KernelEntry>& out);
// Launch form 3 of multi-warp and cluster tiles, attached to the entries
// above (run last).
void register_xc_keys(std::vector<KernelEntry>& out);
void register_xc_rec(std::vector<KernelEntry>& out);
void register_xc_cluster_rec(std::vector<KernelEntry>& out);
void register_xc_u64rec(std::vector<KernelEntry>& out);

const std::vector<KernelEntry>& registry();

struct RaggedCtl;

// The persistent ragged kernel of one element type.
using RaggedLaunch = cudaError_t (*)(const void* in, void* out, const int* d_off, const int* d_ids,
                                     RaggedCtl* ctl, unsigned family_mask, unsigned dedicated_mask, int grid,
                                     cudaStream_t stream);
struct RaggedEntry {
    int dtype;
    int stable;
    int cta;          // threads per CTA
    int nb;           // buckets: W = 8 .. 8 << (nb - 1)
    int lka, lkb;     // log2 elements per thread of shape families A and B
    size_t smem;      // dynamic shared memory bytes
    RaggedLaunch launch;  // family_mask, dedicated_mask: see k_sort_ragged
    int (*resident_per_sm)();  // CTAs per SM (occupancy), 0 on error
};

// TMA-pipelined packed kernels (launch form 2) of single-warp-team tiles.
struct TmaEntry {
    int dtype;
    int stable;
    int lk, lg;
    cudaError_t (*launch)(const void* in, void* out, int n, long long arrays, cudaStream_t stream);
};
const std::vector<TmaEntry>& tma_registry();
int64_t tma_timeouts();  // CTAs of the TMA kernels that gave up waiting for a load
bool tma_set_extra_tx(unsigned int bytes);  // failure-detection test hook

void register_ragged_i32(std::vector<RaggedEntry>& out);
void register_ragged_rec(std::vector<RaggedEntry>& out);
void register_ragged_u64(std::vector<RaggedEntry>& out);

const std::vector<RaggedEntry>& ragged_registry();

// Registry indices of the cluster kernels that sort the ragged working lengths
// first_log2w, first_log2w + 1, ... above the persistent kernel's buckets (at
// most kMaxOverflow of them; idx may be null): for each length the cluster
// tile with the fewest CTAs per array.  Returns how many lengths are covered.
// Plans and the allocation-free ragged sort both use it, so they run the same
// kernels.
int overflow_entries(int dtype, int stable, int first_log2w, int* idx);

}  // namespace b200s
