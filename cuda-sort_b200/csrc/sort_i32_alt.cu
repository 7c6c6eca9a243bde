// int32-key tile alternatives for the tile table, in a translation unit of
// their own so that the library's parallel build is not held up by one unit.
#include "instantiate.cuh"

namespace b200s {

void register_i32_alt(std::vector<KernelEntry>& o) {
    constexpr int D = 0;  // B200S_I32
    // K = 16 alternatives for the tile table.
    o.push_back(Packed<ElemI32, 4, 1, 0>::entry(D));
    o.push_back(Packed<ElemI32, 4, 2, 0>::entry(D));
    o.push_back(Packed<ElemI32, 4, 3, 0>::entry(D));
    o.push_back(Packed<ElemI32, 4, 4, 0>::entry(D));
    o.push_back(Packed<ElemI32, 4, 5, 0>::entry(D));
    o.push_back(Packed<ElemI32, 4, 5, 1>::entry(D));
    o.push_back(Packed<ElemI32, 4, 5, 2>::entry(D));
    // K = 64: ten shuffle layers instead of fifteen for a 1024-key array.
    o.push_back(Packed<ElemI32, 6, 3, 0>::entry(D));
    o.push_back(Packed<ElemI32, 6, 4, 0>::entry(D));
    o.push_back(Packed<ElemI32, 6, 5, 0>::entry(D));
}

}  // namespace b200s
