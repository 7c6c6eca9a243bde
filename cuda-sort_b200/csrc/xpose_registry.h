// Host-side registry of the transposed-network kernels (launch form 3 of
// single-warp tiles; csrc/xpose.cuh).  Kept apart from registry.h so that the
// rest of the library does not depend on it.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace b200s {

struct XposeEntry {
    int dtype;
    int stable;
    int lk, lg;  // the tile shape it serves: K = 2^lk elements per lane, 2^lg lanes per array
    cudaError_t (*launch)(const void* in, void* out, int n, long long arrays, cudaStream_t stream, unsigned opts);
    cudaError_t (*attrs)(cudaFuncAttributes* attr);
    int cta;      // threads per CTA
    size_t smem;  // dynamic shared memory per CTA
    int align;    // the arrays' buffers must be aligned to this many bytes (one element)
    // The same network over a CSR id list (a ragged length class): host count,
    // or count and list position on the device with a work queue.
    cudaError_t (*launch_list)(const void* in, void* out, const int* d_off, const int* d_ids, int count,
                               cudaStream_t stream);
    cudaError_t (*launch_list_dev)(const void* in, void* out, const int* d_off, const int* d_ids,
                                   const int* d_count, const int* d_base, int* d_head, int max_count,
                                   cudaStream_t stream);
};

const std::vector<XposeEntry>& xpose_registry();

}  // namespace b200s
