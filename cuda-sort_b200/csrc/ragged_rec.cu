// Persistent ragged kernels for IntAndData records (reference tie order and
// stable mode): buckets W = 8 .. 8192, families K = 16 (A) and K = 8 (B).
#include "instantiate.cuh"

namespace b200s {

void register_ragged_rec(std::vector<RaggedEntry>& o) {
    o.push_back(Ragged<ElemRecI32, 512, 11, 4, 3>::entry(1));
    o.push_back(Ragged<ElemRecI32S, 512, 11, 4, 3>::entry(1));
}

}  // namespace b200s
