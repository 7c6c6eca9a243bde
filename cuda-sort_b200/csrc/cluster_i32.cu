// Cluster kernels for int32 and uint64 keys: 512-thread CTAs, 2..8 CTAs per
// array (int32: 16384 keys per CTA, W = 32768 .. 131072; uint64: 8192 keys
// per CTA, W = 16384 .. 65536).
#include "instantiate.cuh"

namespace b200s {

void register_cluster_keys(std::vector<KernelEntry>& o) {
    o.push_back(ClusterTile<ElemI32, 5, 5, 4, 1, false>::entry(0));
    o.push_back(ClusterTile<ElemI32, 5, 5, 4, 2, false>::entry(0));
    o.push_back(ClusterTile<ElemI32, 5, 5, 4, 3, false>::entry(0));
    o.push_back(ClusterTile<ElemU64, 4, 5, 4, 1, false>::entry(2));
    o.push_back(ClusterTile<ElemU64, 4, 5, 4, 2, false>::entry(2));
    o.push_back(ClusterTile<ElemU64, 4, 5, 4, 3, false>::entry(2));
}

}  // namespace b200s
