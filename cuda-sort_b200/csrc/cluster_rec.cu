// Cluster kernels for IntAndData records, reference tie order and stable.
//
// 1024-thread CTAs of 16384 records (K = 16, 32 lanes, 32 warps, single-
// buffered shared memory: 128 KB, or 192 KB for the stable records that carry
// their original index; 64 registers): one CTA for W = 16384 and 2 or 4 CTAs
// per array for W = 32768 and 65536.  Against 512-thread CTAs of 8192 records
// this halves the cross-CTA layers, whose distributed-shared-memory reads run
// at about 1/14 of the local shared-memory rate, and 4-CTA clusters place on
// the GPCs better than 8-CTA ones.  Measured on 16 M records (n = 65536 /
// 32768 / 16384): reference order 1.49 / 1.06 / 0.71 -> 1.17 / 0.88 / 0.66 ms,
// stable 3.56 / 2.48 / 1.73 -> 2.30 / 1.43 / 1.21 ms; the output is the same
// network's, bit for bit.
#include "instantiate.cuh"

namespace b200s {

void register_cluster_rec(std::vector<KernelEntry>& o) {
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 5, 0, true>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 5, 1, true>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 5, 2, true>::entry(1));
    // Latency alternatives for a few long arrays (b200s_sort_packed picks them
    // when every array's CTAs fit on the GPU at once): 512-thread CTAs of 8192
    // records, 2..8 per array, half the work per SM.
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 1, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 2, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32, 4, 5, 4, 3, false>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 5, 0, true>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 5, 1, true>::entry(1));
    o.push_back(ClusterTile<ElemRecI32S, 4, 5, 5, 2, true>::entry(1));
}

}  // namespace b200s
