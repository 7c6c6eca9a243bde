// Persistent ragged kernels for IntAndData records (reference tie order and
// stable mode): buckets W = 8 .. 8192, families K = 16 (A) and K = 8 (B).
// Reference tie order: one shared-memory buffer per team and registers sized
// for two CTAs per SM, 32 warps resident instead of 16 (measured 5 % faster
// on 200 000 ragged arrays than double buffering at one CTA per SM).
#include "instantiate.cuh"

namespace b200s {

void register_ragged_rec(std::vector<RaggedEntry>& o) {
    o.push_back(Ragged<ElemRecI32, 512, 11, 4, 3, true, 2>::entry(1));
    o.push_back(Ragged<ElemRecI32S, 512, 11, 4, 3>::entry(1));  // 3 words per element: spills at 64 registers
}

}  // namespace b200s
