// IntAndData record kernels: reference tie order (default) and stable mode.
#include "instantiate.cuh"

namespace b200s {

template <class E>
static void add_rec(std::vector<KernelEntry>& o) {
    constexpr int D = 1;  // B200S_I32_I32
    o.push_back(Packed<E, 3, 0, 0>::entry(D));  // W = 8
    o.push_back(Packed<E, 4, 0, 0>::entry(D));  // W = 16, one lane per array
    o.push_back(Packed<E, 4, 1, 0>::entry(D));
    o.push_back(Packed<E, 4, 2, 0>::entry(D));
    o.push_back(Packed<E, 4, 3, 0>::entry(D));
    o.push_back(Packed<E, 4, 4, 0>::entry(D));
    o.push_back(Packed<E, 4, 5, 0>::entry(D));  // W = 512
    // Multi-warp tiles single-buffer their shared-memory layers: more CTAs
    // per SM (the record kernels are ALU bound, residency hides latency).
    o.push_back(Packed<E, 4, 5, 1, true>::entry(D));  // W = 1024
    o.push_back(Packed<E, 4, 5, 2, true>::entry(D));
    o.push_back(Packed<E, 4, 5, 3, true>::entry(D));
    o.push_back(Packed<E, 4, 5, 4, true>::entry(D));  // W = 8192, 512 threads
}

void register_rec(std::vector<KernelEntry>& o) {
    add_rec<ElemRecI32>(o);
    add_rec<ElemRecI32S>(o);
    // A warp per 1024-record array, 32 records per lane; two 512-record arrays
    // per warp (also the tile of the transposed-network form at W = 512).
    o.push_back(Packed<ElemRecI32, 5, 4, 0>::entry(1));
    o.push_back(Packed<ElemRecI32, 5, 5, 0>::entry(1));
    o.push_back(Packed<ElemRecI32, 5, 5, 1>::entry(1));
    // 32 records per thread for W = 4096 and 8192 (128 and 256 threads): the
    // transposed form needs fewer window moves than with 16 per thread.
    o.push_back(Packed<ElemRecI32, 5, 5, 2, true>::entry(1));
    o.push_back(Packed<ElemRecI32, 5, 5, 3, true>::entry(1));
}

}  // namespace b200s
