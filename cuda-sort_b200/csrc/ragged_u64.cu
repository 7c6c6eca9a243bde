// Persistent ragged kernels for uint64 keys (W = 8 .. 8192, 512 threads) and
// {uint64 key, int32 payload} records (W = 8 .. 4096, 256 threads: their
// 16-byte registers double the shared-memory tile).
#include "instantiate.cuh"

namespace b200s {

void register_ragged_u64(std::vector<RaggedEntry>& o) {
    o.push_back(Ragged<ElemU64, 512, 11, 4, 3>::entry(2));
    o.push_back(Ragged<ElemRecU64, 256, 10, 4, 3>::entry(3));
    o.push_back(Ragged<ElemRecU64S, 256, 10, 4, 3>::entry(3));
}

}  // namespace b200s
