// int32-key kernels (keys alone: the stable flag changes nothing).
#include "instantiate.cuh"

namespace b200s {

void register_i32(std::vector<KernelEntry>& o) {
    constexpr int D = 0;  // B200S_I32
    o.push_back(Packed<ElemI32, 3, 0, 0>::entry(D));  // W = 8, one lane per array
    o.push_back(Packed<ElemI32, 4, 0, 0>::entry(D));  // W = 16
    o.push_back(Packed<ElemI32, 5, 0, 0>::entry(D));  // W = 32
    o.push_back(Packed<ElemI32, 5, 1, 0>::entry(D));
    o.push_back(Packed<ElemI32, 5, 2, 0>::entry(D));
    o.push_back(Packed<ElemI32, 5, 3, 0>::entry(D));
    o.push_back(Packed<ElemI32, 5, 4, 0>::entry(D));
    o.push_back(Packed<ElemI32, 5, 5, 0>::entry(D));  // W = 1024, a warp per array
    o.push_back(Packed<ElemI32, 5, 5, 1>::entry(D));  // W = 2048
    o.push_back(Packed<ElemI32, 5, 5, 2>::entry(D));
    o.push_back(Packed<ElemI32, 5, 5, 3>::entry(D));
    o.push_back(Packed<ElemI32, 5, 5, 4>::entry(D));  // W = 16384, 512 threads
    register_i32_alt(o);  // the alternatives, compiled in their own unit
}

}  // namespace b200s
