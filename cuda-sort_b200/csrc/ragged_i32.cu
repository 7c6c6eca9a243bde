// Persistent ragged kernel for int32 keys: buckets W = 8 .. 16384,
// shape families K = 32 (A) and K = 16 (B), 512 threads per CTA.
#include "instantiate.cuh"

namespace b200s {

void register_ragged_i32(std::vector<RaggedEntry>& o) {
    o.push_back(Ragged<ElemI32, 512, 12, 5, 4>::entry(0));
}

}  // namespace b200s
