// On-chip bandwidth probes for the on-chip roofline of the sort kernels:
// shared memory inside one CTA, and distributed shared memory read across a
// thread-block cluster.  Built as libb200sort_onchip.so and called by the
// benchmark on the device it measures; never linked into the library.
//
// Shared memory: every CTA of a full persistent grid (resident CTAs only)
// streams its own 64 KB buffer with conflict-free 128-bit loads (a warp reads
// 512 consecutive bytes), either reading alone or copying one half of the
// buffer into the other.  Distributed shared memory: every CTA of a cluster
// reads the 64 KB buffer of the next CTA in the cluster the same way
// (cluster.map_shared_rank, read with generic loads), with a cluster barrier
// before the first and after the last remote read.  Bytes counted are the
// bytes each thread loads (and stores, for the copy); the nominal shared
// memory rate is 128 bytes per clock per SM.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace cg = cooperative_groups;

namespace {

constexpr int kThreads = 1024;
constexpr int kChunks = 4096;  // 16-byte chunks per CTA buffer (64 KB)

__device__ __forceinline__ uint4 lds128(const uint4* p) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p)))
                 : "memory");
    return v;
}
__device__ __forceinline__ void sts128(uint4* p, uint4 v) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}
// generic 128-bit load (a distributed-shared-memory address from map_shared_rank)
__device__ __forceinline__ uint4 ld128(const uint4* p) {
    uint4 v;
    asm volatile("ld.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

__device__ __forceinline__ void fill(uint4* buf) {
    for (int i = int(threadIdx.x); i < kChunks; i += blockDim.x)
        buf[i] = make_uint4(unsigned(i), unsigned(i) * 3u, unsigned(i) ^ 0x5555u, ~unsigned(i));
}

// mode 0: read only; mode 1: copy the lower half of the buffer into the upper half
__global__ void __launch_bounds__(kThreads) k_smem(int iters, int mode, uint4* sink) {
    extern __shared__ __align__(16) uint4 buf[];
    fill(buf);
    __syncthreads();
    uint4 acc = make_uint4(0, 0, 0, 0);
    const int t = int(threadIdx.x);
    if (mode == 0) {
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int k = 0; k < kChunks / kThreads; ++k) {
                const uint4 v = lds128(buf + ((t + k * kThreads + it) & (kChunks - 1)));
                acc.x ^= v.x;
                acc.y ^= v.y;
                acc.z ^= v.z;
                acc.w ^= v.w;
            }
        }
    } else {
        constexpr int HALF = kChunks / 2;
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int k = 0; k < HALF / kThreads; ++k) {
                const int i = (t + k * kThreads + it) & (HALF - 1);
                sts128(buf + HALF + i, lds128(buf + i));
            }
        }
        __syncthreads();
        acc = lds128(buf + HALF + t);
    }
    if ((acc.x ^ acc.y ^ acc.z ^ acc.w) == 0x9e3779b9u) sink[blockIdx.x] = acc;  // keeps the loads
}

// Every CTA reads the buffer of CTA (rank + 1) % cluster size.
__global__ void __launch_bounds__(kThreads) k_dsmem(int iters, uint4* sink) {
    extern __shared__ __align__(16) uint4 buf[];
    cg::cluster_group cluster = cg::this_cluster();
    fill(buf);
    cluster.sync();
    const unsigned peer = (cluster.block_rank() + 1) % cluster.num_blocks();
    const uint4* remote = cluster.map_shared_rank(buf, int(peer));
    uint4 acc = make_uint4(0, 0, 0, 0);
    const int t = int(threadIdx.x);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < kChunks / kThreads; ++k) {
            const uint4 v = ld128(remote + ((t + k * kThreads + it) & (kChunks - 1)));
            acc.x ^= v.x;
            acc.y ^= v.y;
            acc.z ^= v.z;
            acc.w ^= v.w;
        }
    }
    cluster.sync();  // no CTA leaves while a peer still reads its buffer
    if ((acc.x ^ acc.y ^ acc.z ^ acc.w) == 0x9e3779b9u) sink[blockIdx.x] = acc;
}

constexpr size_t kSmem = size_t(kChunks) * 16;

int time_launch(float* ms, const cudaLaunchConfig_t& cfg, void (*fn)(int, int, uint4*), int iters, int mode,
                uint4* sink) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return 1;
    cudaLaunchKernelEx(&cfg, fn, iters, mode, sink);  // warm-up
    cudaEventRecord(a, cfg.stream);
    cudaLaunchKernelEx(&cfg, fn, iters, mode, sink);
    cudaEventRecord(b, cfg.stream);
    const cudaError_t e = cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

extern "C" {

// Shared-memory bandwidth of the whole device in GB/s: loads alone (read_gbs)
// and load + store copies (copy_gbs, bytes loaded plus bytes stored).
// Returns 0 on success.
int onchip_smem_gbs(int device, double* read_gbs, double* copy_gbs) {
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 1;
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(k_smem), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kSmem)) != cudaSuccess)
        return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_smem, kThreads, kSmem) != cudaSuccess ||
        per_sm < 1)
        return 1;
    const int grid = sms * per_sm;
    uint4* sink = nullptr;
    if (cudaMalloc(&sink, size_t(grid) * sizeof(uint4)) != cudaSuccess) return 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kSmem;
    cfg.stream = nullptr;
    const int iters = 2000;
    float ms = 0.f;
    int rc = time_launch(&ms, cfg, k_smem, iters, 0, sink);
    if (!rc) *read_gbs = double(grid) * kThreads * 16.0 * (kChunks / kThreads) * iters / (ms * 1e-3) / 1e9;
    if (!rc) rc = time_launch(&ms, cfg, k_smem, iters, 1, sink);
    if (!rc) *copy_gbs = double(grid) * kThreads * 32.0 * (kChunks / 2 / kThreads) * iters / (ms * 1e-3) / 1e9;
    cudaFree(sink);
    return rc;
}

// Distributed-shared-memory read bandwidth of the whole device in GB/s with
// clusters of `cluster` CTAs (2..8), each CTA reading a peer's buffer.
int onchip_dsmem_gbs(int device, int cluster, double* read_gbs) {
    if (cluster < 2 || cluster > 8 || (cluster & (cluster - 1))) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(k_dsmem), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kSmem)) != cudaSuccess)
        return 1;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = unsigned(cluster);
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(cluster));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kSmem;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_dsmem, &cfg) != cudaSuccess || clusters < 1) return 1;
    cfg.gridDim = dim3(unsigned(clusters * cluster));
    uint4* sink = nullptr;
    if (cudaMalloc(&sink, size_t(clusters) * cluster * sizeof(uint4)) != cudaSuccess) return 1;
    const int iters = 1000;
    cudaEvent_t a, b;
    int rc = 1;
    if (cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess) {
        cudaLaunchKernelEx(&cfg, k_dsmem, iters, sink);
        cudaEventRecord(a, nullptr);
        cudaLaunchKernelEx(&cfg, k_dsmem, iters, sink);
        cudaEventRecord(b, nullptr);
        float ms = 0.f;
        if (cudaEventSynchronize(b) == cudaSuccess && cudaGetLastError() == cudaSuccess &&
            cudaEventElapsedTime(&ms, a, b) == cudaSuccess) {
            *read_gbs = double(clusters) * cluster * kThreads * 16.0 * (kChunks / kThreads) * iters / (ms * 1e-3) / 1e9;
            rc = 0;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    cudaFree(sink);
    return rc;
}

}  // extern "C"
