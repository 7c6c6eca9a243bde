// Launch form 3 of the multi-warp IntAndData record tiles (reference tie
// order and stable): the transposed network of cta_xpose.cuh, one array per
// CTA.  MINB: 64 registers per thread for the 8-byte records, 128 for the
// stable ones (which carry their original position).
#include "instantiate_xc.cuh"

namespace b200s {

void register_xc_rec(std::vector<KernelEntry>& o) {
    PackedXc<ElemRecI32, 4, 1, 16>::attach_to(o, 1);  // W = 1024
    PackedXc<ElemRecI32, 4, 2, 8>::attach_to(o, 1);
    PackedXc<ElemRecI32, 4, 3, 4>::attach_to(o, 1);
    PackedXc<ElemRecI32, 4, 4, 2>::attach_to(o, 1);   // W = 8192
    PackedXc<ElemRecI32, 5, 1, 8>::attach_to(o, 1);   // W = 2048, 32 records per thread
    PackedXc<ElemRecI32, 5, 2, 4>::attach_to(o, 1);   // W = 4096
    PackedXc<ElemRecI32, 5, 3, 2>::attach_to(o, 1);   // W = 8192
    PackedXc<ElemRecI32S, 4, 1, 8>::attach_to(o, 1);
    PackedXc<ElemRecI32S, 4, 2, 4>::attach_to(o, 1);
    PackedXc<ElemRecI32S, 4, 3, 2>::attach_to(o, 1);
    PackedXc<ElemRecI32S, 4, 4, 1>::attach_to(o, 1);
}

}  // namespace b200s
