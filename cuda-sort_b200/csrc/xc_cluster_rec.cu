// Launch form 3 of the IntAndData record cluster tiles: the transposed
// network of cta_xpose.cuh (1024-thread CTAs of 16384 records, and the
// 512-thread latency alternatives).
#include "instantiate_xc.cuh"

namespace b200s {

void register_xc_cluster_rec(std::vector<KernelEntry>& o) {
    ClusterXc<ElemRecI32, 4, 5, 5, 0, true>::attach_to(o, 1);
    ClusterXc<ElemRecI32, 4, 5, 5, 1, true>::attach_to(o, 1);
    ClusterXc<ElemRecI32, 4, 5, 5, 2, true>::attach_to(o, 1);
    ClusterXc<ElemRecI32, 4, 5, 4, 1, false>::attach_to(o, 1);
    ClusterXc<ElemRecI32, 4, 5, 4, 2, false>::attach_to(o, 1);
    ClusterXc<ElemRecI32, 4, 5, 4, 3, false>::attach_to(o, 1);
    ClusterXc<ElemRecI32S, 4, 5, 5, 0, true>::attach_to(o, 1);
    ClusterXc<ElemRecI32S, 4, 5, 5, 1, true>::attach_to(o, 1);
    ClusterXc<ElemRecI32S, 4, 5, 5, 2, true>::attach_to(o, 1);
}

}  // namespace b200s
