// Cluster kernels for IntAndData records (reference tie order and stable
// mode): 512-thread CTAs of 8192 records, 2..8 CTAs per array
// (W = 16384 .. 65536).  The 8-CTA reference-order kernel uses single-buffered
// shared memory and 64 registers so that two CTAs share an SM: one 8-CTA
// cluster per SM set leaves 28 of 148 SMs idle (15 clusters resident), two
// per SM place 30.  Measured on 256 x 65536 records: 1.51 -> 1.48 ms; the 2-
// and 4-CTA kernels are 7-10 % slower that way (spills, extra barriers) and
// stay double-buffered.
#include "instantiate.cuh"

namespace b200s {

void register_cluster_rec(std::vector<KernelEntry>& o) {
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 1, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 2, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 3, true, 2>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 4, 1, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 4, 2, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 4, 3, false>::entry(1));
}

}  // namespace b200s
