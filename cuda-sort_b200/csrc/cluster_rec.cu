// Cluster kernels for IntAndData records (reference tie order and stable
// mode): 512-thread CTAs of 8192 records, 2..8 CTAs per array
// (W = 16384 .. 65536).
#include "instantiate.cuh"

namespace b200s {

void register_cluster_rec(std::vector<KernelEntry>& o) {
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 1, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 2, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 3, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 4, 1, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 4, 2, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 4, 3, false>::entry(1));
}

}  // namespace b200s
