// TMA-pipelined packed kernels (tma.cuh) for the single-warp-team tiles, and
// their launcher: tensor-map encoding (cached per buffer and shape) and the
// persistent grid.  Launch form 2 of a tile; the C ABI falls back to the
// one-shot kernel when the batch does not meet the TMA requirements.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "registry.h"
#include "tma.cuh"

namespace b200s {

namespace {

constexpr int kDepth = 3;

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor {32 words, rows, arrays} over a packed batch, box {32, rows, apc}.
bool encode(CUtensorMap* m, const void* base, int rows, long long arrays, int apc) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {32, cuuint64_t(rows), cuuint64_t(arrays)};
    const cuuint64_t strides[2] = {128, cuuint64_t(rows) * 128};
    const cuuint32_t box[3] = {32, cuuint32_t(rows), cuuint32_t(apc)};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Small cache of encoded maps: callers that alternate between a few buffers
// (double buffering, benchmark rotations) pay for the encoding once.
struct MapKey {
    const void* base;
    int rows;
    long long arrays;
    int apc;
    bool operator==(const MapKey& o) const {
        return base == o.base && rows == o.rows && arrays == o.arrays && apc == o.apc;
    }
};
std::mutex g_map_mutex;
std::vector<std::pair<MapKey, CUtensorMap>> g_maps;
size_t g_next = 0;
constexpr size_t kMapCache = 32;

bool get_map(CUtensorMap* out, const void* base, int rows, long long arrays, int apc) {
    const MapKey k{base, rows, arrays, apc};
    std::lock_guard<std::mutex> lk(g_map_mutex);
    for (const auto& e : g_maps)
        if (e.first == k) {
            *out = e.second;
            return true;
        }
    CUtensorMap m;
    if (!encode(&m, base, rows, arrays, apc)) return false;
    if (g_maps.size() < kMapCache) g_maps.push_back({k, m});
    else g_maps[g_next++ % kMapCache] = {k, m};
    *out = m;
    return true;
}

__device__ TmaStatus g_tma_status;

TmaStatus* status_ptr() {
    static std::atomic<TmaStatus*> per_dev[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    TmaStatus* p = per_dev[dev & 63].load();
    if (!p) {
        void* a = nullptr;
        if (cudaGetSymbolAddress(&a, g_tma_status) != cudaSuccess) return nullptr;
        p = static_cast<TmaStatus*>(a);
        per_dev[dev & 63].store(p);
    }
    return p;
}

template <class E, int LK, int LG, int CTA>
struct PackedTma {
    using S = Shape<LK, LG, 0>;
    static constexpr int APC = CTA / S::TPA;

    static size_t smem_bytes(int rows) {
        return size_t(kDepth) * ((size_t(APC) * rows * 128 + 1023) & ~size_t(1023)) + 1024;
    }
    // One CTA per SM-slot, no more than there are chunks (cached per device
    // and shared-memory size).
    static cudaError_t launch(const void* in, void* out, int n, long long arrays, cudaStream_t st) {
        auto fn = k_sort_packed_tma<E, S, CTA, kDepth>;
        const int rows = n * int(sizeof(typename E::Mem)) / 128;
        if (rows < 1 || rows > 256) return cudaErrorInvalidValue;
        const size_t smem = smem_bytes(rows);
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        // resident CTAs for this shared-memory size, per device (the
        // attribute is set on first use)
        // The shared-memory opt-in is one value per kernel and device: set it
        // once to the largest array this tile covers (W elements), so that
        // launches for shorter arrays never lower it under a longer one.
        static std::atomic<int> opted[64];
        if (!opted[dev & 63].load(std::memory_order_acquire)) {
            const int max_rows = S::W * int(sizeof(typename E::Mem)) / 128;
            e = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(smem_bytes(max_rows > 0 ? max_rows : 1)));
            if (e != cudaSuccess) return e;
            opted[dev & 63].store(1, std::memory_order_release);
        }
        if (rows * 128 > S::W * int(sizeof(typename E::Mem))) return cudaErrorInvalidValue;
        static std::atomic<int> resident[64][257];
        int cap = resident[dev & 63][rows].load(std::memory_order_relaxed);
        if (cap == 0) {
            int per_sm = 0, sms = 0;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, CTA, smem)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if (per_sm <= 0) return cudaErrorInvalidConfiguration;
            cap = per_sm * sms;
            resident[dev & 63][rows].store(cap, std::memory_order_relaxed);
        }
        CUtensorMap tin, tout;
        if (!get_map(&tin, in, rows, arrays, APC) || !get_map(&tout, out, rows, arrays, APC))
            return cudaErrorInvalidValue;
        TmaStatus* status = status_ptr();
        if (!status) return cudaErrorInvalidSymbol;
        const long long chunks = (arrays + APC - 1) / APC;
        const long long grid = std::min<long long>(chunks, cap);
        // programmatic dependent launch (the kernel waits for the stream's
        // previous kernel before its first access)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(grid));
        cfg.blockDim = dim3(CTA);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr.val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, fn, tin, tout, n, arrays, rows, status);
    }
    static TmaEntry entry(int dtype) { return TmaEntry{dtype, E::kStable ? 1 : 0, LK, LG, &launch}; }
};

}  // namespace

void register_tma(std::vector<TmaEntry>& o) {
    // int32 keys
    o.push_back(PackedTma<ElemI32, 5, 5, 128>::entry(0));  // W = 1024, a warp per array
    o.push_back(PackedTma<ElemI32, 5, 4, 128>::entry(0));  // W = 512
    o.push_back(PackedTma<ElemI32, 4, 5, 128>::entry(0));  // W = 512, K = 16
    o.push_back(PackedTma<ElemI32, 5, 3, 128>::entry(0));  // W = 256
    o.push_back(PackedTma<ElemI32, 5, 2, 128>::entry(0));  // W = 128
    o.push_back(PackedTma<ElemI32, 5, 0, 128>::entry(0));  // W = 32
    // IntAndData records (reference tie order)
    o.push_back(PackedTma<ElemRecI32, 4, 1, 64>::entry(1));  // W = 32
    o.push_back(PackedTma<ElemRecI32, 4, 2, 64>::entry(1));  // W = 64
    o.push_back(PackedTma<ElemRecI32, 4, 3, 64>::entry(1));  // W = 128
    o.push_back(PackedTma<ElemRecI32, 4, 4, 64>::entry(1));  // W = 256
    o.push_back(PackedTma<ElemRecI32, 4, 5, 64>::entry(1));  // W = 512
    o.push_back(PackedTma<ElemRecI32, 5, 5, 64>::entry(1));  // W = 1024
}

const std::vector<TmaEntry>& tma_registry() {
    static std::vector<TmaEntry> all = [] {
        std::vector<TmaEntry> v;
        register_tma(v);
        return v;
    }();
    return all;
}

bool tma_set_extra_tx(unsigned int bytes) {
    TmaStatus* p = status_ptr();
    return p && cudaMemcpy(&p->extra_tx, &bytes, sizeof(bytes), cudaMemcpyHostToDevice) == cudaSuccess;
}

int64_t tma_timeouts() {
    TmaStatus s{};
    if (cudaMemcpyFromSymbol(&s, g_tma_status, sizeof(s)) != cudaSuccess) return -1;
    return int64_t(s.timeouts);
}

}  // namespace b200s
