// Transposed-network kernels (launch form 3): every comparator layer in
// registers, the tile re-laid out through shared memory between windows
// (xpose.cuh).  Keys (int32, uint64) read their arrays with coalesced striped
// accesses (their input order is unobservable); IntAndData records load
// coalesced through the shared region, keeping their order (the reference's
// tie order depends on it).  Both store coalesced through the shared region.
#include <algorithm>
#include <atomic>

#include "xpose.cuh"
#include "xpose_registry.h"

namespace b200s {

namespace {

// One warp per CTA (arrays are independent per warp, no CTA barrier).  MINB
// bounds the registers: 28 warps per SM for int32 keys (48 registers: a
// 4096-array batch in one wave on 148 SMs); records and 64-bit keys hold twice
// the data per element (16 warps per SM at 32 per lane, 24 at 16).
template <class E, int LK, int LG, int IO, int MINB_ = 28>
struct Xpose {
    static constexpr int WPC = 1, MINB = MINB_;
    static constexpr int APW = 32 >> LG;
    static constexpr size_t SMEM = size_t(WPC) * APW * xp_region<LK, LG>() * sizeof(typename E::Reg);
    static constexpr auto kernel() { return k_sort_xpose<E, LK, LG, WPC, MINB, IO>; }

    // Programmatic dependent launch: the grid may be scheduled while the
    // stream's previous kernel drains; the kernel waits for that kernel's
    // completion before its first access (griddepcontrol.wait).
    static cudaError_t launch(const void* in, void* out, int n, long long arrays, cudaStream_t st, unsigned opts) {
        const long long per_cta = (long long)WPC * APW;
        const long long grid = std::min<long long>((arrays + per_cta - 1) / per_cta, 0x7fffffffLL);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(grid));
        cfg.blockDim = dim3(WPC * 32);
        cfg.dynamicSmemBytes = SMEM;
        cfg.stream = st;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr.val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, kernel(), static_cast<const typename E::Mem*>(in),
                                  static_cast<typename E::Mem*>(out), n, arrays, opts);
    }
    static cudaError_t attrs(cudaFuncAttributes* a) {
        return cudaFuncGetAttributes(a, reinterpret_cast<const void*>(kernel()));
    }
    static constexpr auto list_kernel() { return k_sort_xpose_list<E, LK, LG, MINB, IO>; }
    static cudaError_t launch_list(const void* in, void* out, const int* off, const int* ids, int count,
                                   cudaStream_t st) {
        const int grid = std::max(1, (count + APW - 1) / APW);
        list_kernel()<<<dim3(unsigned(grid)), dim3(32), SMEM, st>>>(static_cast<const typename E::Mem*>(in),
                                                                   static_cast<typename E::Mem*>(out), off, ids,
                                                                   count, nullptr, nullptr, nullptr);
        return cudaGetLastError();
    }
    // Resident warps (cached per device), at most what max_count arrays need,
    // pulling arrays from the queue.
    static cudaError_t launch_list_dev(const void* in, void* out, const int* off, const int* ids, const int* d_count,
                                       const int* d_base, int* d_head, int max_count, cudaStream_t st) {
        static std::atomic<int> resident[64];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        int cap = resident[dev & 63].load(std::memory_order_relaxed);
        if (cap == 0) {
            int per_sm = 0, sms = 0;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, list_kernel(), 32, SMEM)) != cudaSuccess)
                return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            cap = per_sm * sms;
            if (cap <= 0) return cudaErrorInvalidConfiguration;
            resident[dev & 63].store(cap, std::memory_order_relaxed);
        }
        const int need = std::max(1, (max_count + APW - 1) / APW);
        list_kernel()<<<dim3(unsigned(std::min(need, cap))), dim3(32), SMEM, st>>>(
            static_cast<const typename E::Mem*>(in), static_cast<typename E::Mem*>(out), off, ids, 0, d_count, d_base,
            d_head);
        return cudaGetLastError();
    }
    static XposeEntry entry(int dtype) {
        return XposeEntry{dtype,    E::kStable ? 1 : 0, LK,   LG, &launch, &attrs, WPC * 32, SMEM,
                          int(sizeof(typename E::Mem)), &launch_list, &launch_list_dev};
    }
};

}  // namespace

const std::vector<XposeEntry>& xpose_registry() {
    static const std::vector<XposeEntry> all = [] {
        std::vector<XposeEntry> v;
        constexpr int I32 = 0;                              // B200S_I32
        v.push_back(Xpose<ElemI32, 5, 5, kXpIoStriped>::entry(I32));  // W = 1024, a warp per array
        v.push_back(Xpose<ElemI32, 5, 4, kXpIoStriped>::entry(I32));  // W = 512, two arrays per warp
        v.push_back(Xpose<ElemI32, 5, 3, kXpIoStriped>::entry(I32));  // W = 256, four arrays per warp
        constexpr int REC = 1;                                     // B200S_I32_I32, reference tie order
        v.push_back(Xpose<ElemRecI32, 5, 5, kXpIoStaged, 16>::entry(REC));  // W = 1024
        v.push_back(Xpose<ElemRecI32, 5, 4, kXpIoStaged, 16>::entry(REC));  // W = 512
        v.push_back(Xpose<ElemRecI32, 4, 4, kXpIoStaged, 24>::entry(REC));  // W = 256
        v.push_back(Xpose<ElemRecI32, 4, 3, kXpIoStaged, 24>::entry(REC));  // W = 128
        v.push_back(Xpose<ElemRecI32, 4, 2, kXpIoStaged, 24>::entry(REC));  // W = 64
        // stable records: (key, data, position) registers, 16 per lane
        v.push_back(Xpose<ElemRecI32S, 4, 4, kXpIoStaged, 20>::entry(REC));  // W = 256
        v.push_back(Xpose<ElemRecI32S, 4, 3, kXpIoStaged, 20>::entry(REC));  // W = 128
        v.push_back(Xpose<ElemRecI32S, 4, 2, kXpIoStaged, 20>::entry(REC));  // W = 64
        constexpr int U64 = 2;                                     // B200S_U64
        v.push_back(Xpose<ElemU64, 5, 5, kXpIoStriped, 16>::entry(U64));    // W = 1024
        v.push_back(Xpose<ElemU64, 5, 4, kXpIoStriped, 16>::entry(U64));    // W = 512
        v.push_back(Xpose<ElemU64, 4, 4, kXpIoStriped, 24>::entry(U64));    // W = 256
        v.push_back(Xpose<ElemU64, 4, 3, kXpIoStriped, 24>::entry(U64));    // W = 128
        v.push_back(Xpose<ElemU64, 4, 2, kXpIoStriped, 24>::entry(U64));    // W = 64
        return v;
    }();
    return all;
}

}  // namespace b200s
