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
};

const std::vector<XposeEntry>& xpose_registry();

}  // namespace b200s
