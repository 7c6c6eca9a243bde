// Launch form 3 of the {uint64 key, int32 payload} record tiles: the
// transposed network of cta_xpose.cuh for the multi-warp tiles (W up to
// 4096) and the 8192-record-per-CTA cluster tiles (W up to 65536).
#include "instantiate_xc.cuh"

namespace b200s {

void register_xc_u64rec(std::vector<KernelEntry>& o) {
    PackedXc<ElemRecU64, 4, 1, 8>::attach_to(o, 3);
    PackedXc<ElemRecU64, 4, 2, 4>::attach_to(o, 3);
    PackedXc<ElemRecU64, 4, 3, 2>::attach_to(o, 3);
    PackedXc<ElemRecU64S, 4, 1, 8>::attach_to(o, 3);
    PackedXc<ElemRecU64S, 4, 2, 4>::attach_to(o, 3);
    PackedXc<ElemRecU64S, 4, 3, 2>::attach_to(o, 3);
    ClusterXc<ElemRecU64, 4, 5, 4, 0, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64, 4, 5, 4, 1, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64, 4, 5, 4, 2, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64, 4, 5, 4, 3, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64S, 4, 5, 4, 0, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64S, 4, 5, 4, 1, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64S, 4, 5, 4, 2, true>::attach_to(o, 3);
    ClusterXc<ElemRecU64S, 4, 5, 4, 3, true>::attach_to(o, 3);
}

}  // namespace b200s
