// Cluster kernels for int32 and uint64 keys.  int32: 512-thread CTAs of 16384
// keys, 2..8 CTAs per array (W = 32768 .. 131072), the 4- and 8-CTA tiles
// through the compact network (ElemI32C: the unrolled one spills there).  uint64: 1024-thread
// CTAs of 16384 keys (128 KB of single-buffered shared memory), 1..4 CTAs per
// array (W = 16384 .. 65536): half the cross-CTA layers of 512-thread CTAs of
// 8192 keys (16 M keys, n = 65536: 1.68 -> 1.37 ms; 32768: 1.22 -> 1.02 ms).
#include "instantiate.cuh"

namespace b200s {

void register_cluster_keys(std::vector<KernelEntry>& o) {
    o.push_back(ClusterTile<ElemI32, 5, 5, 4, 1, false>::entry(0));
    o.push_back(ClusterTile<ElemI32C, 5, 5, 4, 2, false>::entry(0));
    o.push_back(ClusterTile<ElemI32C, 5, 5, 4, 3, false>::entry(0));
    o.push_back(ClusterTile<ElemU64, 4, 5, 5, 0, true>::entry(2));
    o.push_back(ClusterTile<ElemU64, 4, 5, 5, 1, true>::entry(2));
    o.push_back(ClusterTile<ElemU64, 4, 5, 5, 2, true>::entry(2));
}

}  // namespace b200s
