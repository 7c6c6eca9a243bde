// Launch form 3 of the multi-warp and cluster tiles of int32 and uint64 keys:
// the transposed network of cta_xpose.cuh (one array per CTA or cluster).
// MINB keeps every tile at 64 registers per thread or fewer.
#include "instantiate_xc.cuh"

namespace b200s {

void register_xc_keys(std::vector<KernelEntry>& o) {
    PackedXc<ElemI32, 5, 1, 8>::attach_to(o, 0);  // W = 2048
    PackedXc<ElemI32, 5, 2, 4>::attach_to(o, 0);
    PackedXc<ElemI32, 5, 3, 2>::attach_to(o, 0);
    PackedXc<ElemI32, 5, 4, 1>::attach_to(o, 0);  // W = 16384
    ClusterXc<ElemI32, 5, 5, 4, 1, false>::attach_to(o, 0);
    ClusterXc<ElemI32, 5, 5, 4, 2, false>::attach_to(o, 0);
    ClusterXc<ElemI32, 5, 5, 4, 3, false>::attach_to(o, 0);
    PackedXc<ElemU64, 4, 1, 16>::attach_to(o, 2);  // W = 1024
    PackedXc<ElemU64, 4, 2, 8>::attach_to(o, 2);
    PackedXc<ElemU64, 4, 3, 4>::attach_to(o, 2);
    PackedXc<ElemU64, 4, 4, 2>::attach_to(o, 2);  // W = 8192
    ClusterXc<ElemU64, 4, 5, 5, 0, true>::attach_to(o, 2);
    ClusterXc<ElemU64, 4, 5, 5, 1, true>::attach_to(o, 2);
    ClusterXc<ElemU64, 4, 5, 5, 2, true>::attach_to(o, 2);
}

}  // namespace b200s
