// Cluster kernels for {uint64 key, int32 payload} records: their 16-byte
// registers use single-buffered shared memory (128 KB per CTA of 8192), one
// to eight CTAs per array (W = 8192 .. 65536).
#include "instantiate.cuh"

namespace b200s {

void register_cluster_u64rec(std::vector<KernelEntry>& o) {
    o.push_back(ClusterTile<ElemRecU64, 4, 5, 4, 0, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64, 4, 5, 4, 1, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64, 4, 5, 4, 2, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64, 4, 5, 4, 3, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64S, 4, 5, 4, 0, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64S, 4, 5, 4, 1, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64S, 4, 5, 4, 2, true>::entry(3));
    o.push_back(ClusterTile<ElemRecU64S, 4, 5, 4, 3, true>::entry(3));
}

}  // namespace b200s
