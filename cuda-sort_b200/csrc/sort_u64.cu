// uint64-key kernels and {uint64 key, int32 payload} record kernels.
#include "instantiate.cuh"

namespace b200s {

template <class E, int D, int MAXLW>
static void add_k16(std::vector<KernelEntry>& o) {
    o.push_back(Packed<E, 3, 0, 0>::entry(D));
    o.push_back(Packed<E, 4, 0, 0>::entry(D));
    o.push_back(Packed<E, 4, 1, 0>::entry(D));
    o.push_back(Packed<E, 4, 2, 0>::entry(D));
    o.push_back(Packed<E, 4, 3, 0>::entry(D));
    o.push_back(Packed<E, 4, 4, 0>::entry(D));
    o.push_back(Packed<E, 4, 5, 0>::entry(D));
    o.push_back(Packed<E, 4, 5, 1>::entry(D));
    o.push_back(Packed<E, 4, 5, 2>::entry(D));
    o.push_back(Packed<E, 4, 5, 3>::entry(D));
    if constexpr (MAXLW >= 4) o.push_back(Packed<E, 4, 5, 4>::entry(D));
}

void register_u64(std::vector<KernelEntry>& o) {
    add_k16<ElemU64, 2, 4>(o);       // W up to 8192
    // 32 keys per lane, a warp per 1024-key array or two 512-key arrays per
    // warp (also the tiles of the transposed-network form at those lengths)
    o.push_back(Packed<ElemU64, 5, 4, 0>::entry(2));
    o.push_back(Packed<ElemU64, 5, 5, 0>::entry(2));
    add_k16<ElemRecU64, 3, 3>(o);    // 16-byte registers: W up to 4096
    add_k16<ElemRecU64S, 3, 3>(o);
}

}  // namespace b200s
