// Transposed-network kernels (launch form 3): every comparator layer in
// registers, the tile re-laid out through shared memory between windows
// (xpose.cuh).  int32 keys read and write their arrays with coalesced, striped
// accesses (their input order is unobservable).
#include <algorithm>

#include "xpose.cuh"
#include "xpose_registry.h"

namespace b200s {

namespace {

// One warp per CTA (arrays are independent per warp, no CTA barrier), at most
// 48 registers so that 28 warps per SM (a 4096-array batch in one wave on 148
// SMs) are resident.
template <class E, int LK, int LG, bool STRIPED>
struct Xpose {
    static constexpr int WPC = 1, MINB = 28;
    static constexpr int APW = 32 >> LG;
    static constexpr size_t SMEM = size_t(WPC) * APW * xp_region<LK, LG>() * sizeof(typename E::Reg);
    static constexpr auto kernel() { return k_sort_xpose<E, LK, LG, WPC, MINB, STRIPED>; }

    static cudaError_t launch(const void* in, void* out, int n, long long arrays, cudaStream_t st, unsigned opts) {
        const long long per_cta = (long long)WPC * APW;
        const long long grid = std::min<long long>((arrays + per_cta - 1) / per_cta, 0x7fffffffLL);
        kernel()<<<dim3(unsigned(grid)), dim3(WPC * 32), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), n, arrays, opts);
        return cudaGetLastError();
    }
    static cudaError_t attrs(cudaFuncAttributes* a) {
        return cudaFuncGetAttributes(a, reinterpret_cast<const void*>(kernel()));
    }
    static XposeEntry entry(int dtype) {
        return XposeEntry{dtype, E::kStable ? 1 : 0, LK, LG, &launch, &attrs, WPC * 32, SMEM};
    }
};

}  // namespace

const std::vector<XposeEntry>& xpose_registry() {
    static const std::vector<XposeEntry> all = [] {
        std::vector<XposeEntry> v;
        constexpr int I32 = 0;                              // B200S_I32
        v.push_back(Xpose<ElemI32, 5, 5, true>::entry(I32));  // W = 1024, a warp per array
        v.push_back(Xpose<ElemI32, 5, 4, true>::entry(I32));  // W = 512, two arrays per warp
        v.push_back(Xpose<ElemI32, 5, 3, true>::entry(I32));  // W = 256, four arrays per warp
        return v;
    }();
    return all;
}

}  // namespace b200s
