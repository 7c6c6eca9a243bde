// Host-side registry of compiled sort kernels (one entry per tile shape and
// element type).  Each translation unit that instantiates kernels appends its
// entries; the C ABI picks one by (dtype, stable, working length).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace b200s {

using PackedLaunch = cudaError_t (*)(const void* in, void* out, int n, long long arrays,
                                     long long grid, cudaStream_t stream);
using AttrQuery = cudaError_t (*)(cudaFuncAttributes* attr);
// Launch over an explicit list of array starts (ragged batches).
using ListLaunch = cudaError_t (*)(const void* in, void* out, const long long* d_start,
                                   const int* d_len, const int* d_ids, long long count,
                                   long long grid, cudaStream_t stream);

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
};

void register_i32(std::vector<KernelEntry>& out);
void register_rec(std::vector<KernelEntry>& out);
void register_u64(std::vector<KernelEntry>& out);

const std::vector<KernelEntry>& registry();

}  // namespace b200s
