// Packed batches streamed through shared memory by the Tensor Memory
// Accelerator: a persistent, pipelined form of the single-warp-team tiles.
//
// The batch is described to TMA as a 3-D tensor of 32-bit words,
// {32 words (one 128-byte row), rows = n*sizeof(elem)/128, arrays}, so that a
// chunk of APC consecutive arrays is one box {32, rows, APC}.  Each CTA
// walks chunks blockIdx.x, blockIdx.x + gridDim.x, ...; one thread keeps
// DEPTH-1 loads in flight (cp.async.bulk.tensor with mbarrier completion)
// while the CTA sorts the current chunk, and returns each sorted chunk with
// a TMA store from the buffer it arrived in.  HBM traffic of later and
// earlier chunks therefore overlaps the comparator layers of the current one,
// which the one-shot kernels (load, sort, store in lock step over a single
// wave) cannot do.
//
// Shared memory uses the 128-byte swizzle: the 16-byte chunk c of 128-byte
// row r is stored at chunk c ^ (r & 7), so that threads reading their own
// consecutive rows hit distinct banks.  Loads carry no multicast.
//
// Requirements, checked on the host: n*sizeof(elem) a multiple of 128 and at
// most 256 rows, 16-byte aligned buffers, a tile of whole-warp teams without
// shared-memory layers (log2_warps = 0).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "network.cuh"

namespace b200s {

namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Load box {c0, c1, c2} of the tensor into shared memory (no multicast).
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void store_3d(const CUtensorMap* map, int c0, int c1, int c2, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src))
                 : "memory");
}

__device__ __forceinline__ void commit_group() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until at most N bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void wait_group_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void wait_group_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Byte offset of 16-byte chunk `col` of 128-byte row `row` in a buffer
// written by a 128-byte-swizzled TMA copy (the buffer is 1024-byte aligned).
__device__ __forceinline__ uint32_t swz(uint32_t row, uint32_t col) { return row * 128u + ((col ^ (row & 7u)) << 4); }

// Clock cycles a thread waits for a chunk before the CTA gives up (~1 s).
constexpr long long kWaitLimit = 2000000000LL;

}  // namespace tma

// Counts CTAs that gave up waiting for a TMA load (0 in a healthy run).
// extra_tx is a test hook: bytes added to every load's expected transaction
// count, so that no chunk ever completes and the bounded wait runs out
// (0 outside the failure-detection test).
struct TmaStatus {
    unsigned long long timeouts;
    unsigned int extra_tx;
    unsigned int reserved;
};

template <class E, class S, int CTA, int DEPTH>
__global__ void __launch_bounds__(CTA) k_sort_packed_tma(const __grid_constant__ CUtensorMap tin,
                                                         const __grid_constant__ CUtensorMap tout, int n,
                                                         long long arrays, int rows, TmaStatus* status) {
    using R = typename E::Reg;
    using M = typename E::Mem;
    static_assert(S::LW == 0, "single-warp teams");
    static_assert(CTA % S::TPA == 0, "whole teams per CTA");
    constexpr int APC = CTA / S::TPA;
    constexpr int EB = int(sizeof(M));
    constexpr int PER = 16 / EB;             // elements per 16-byte chunk
    constexpr int CH = S::K * EB / 16;       // 16-byte chunks per thread
    static_assert(S::K * EB % 16 == 0 && EB <= 16, "whole 16-byte chunks per thread");

    extern __shared__ __align__(1024) unsigned char tma_smem[];
    __shared__ __align__(8) uint64_t full[DEPTH];

    // programmatic dependent launch: the stream's previous kernel has
    // completed before any access (immediate without such a predecessor)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int tid = int(threadIdx.x);
    const int slot = tid / S::TPA;
    const int t = tid % S::TPA;
    const uint32_t buf_bytes = (uint32_t(APC * rows * 128) + 1023u) & ~1023u;
    const uint32_t box_bytes = uint32_t(APC * rows * 128) + status->extra_tx;
    const long long chunks = (arrays + APC - 1) / APC;
    const int valid_chunks = (n * EB) / 16;  // 16-byte chunks of one array
    // 1024-byte aligned base for the swizzle pattern
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tma_smem) + 1023u) & ~uintptr_t(1023u));

    if (tid == 0) {
        for (int d = 0; d < DEPTH; ++d) tma::mbar_init(&full[d], 1);
        tma::fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int d = 0; d < DEPTH - 1; ++d) {
            const long long c = blockIdx.x + (long long)d * gridDim.x;
            if (c >= chunks) break;
            tma::mbar_expect_tx(&full[d], box_bytes);
            tma::load_3d(base + d * buf_bytes, &tin, 0, 0, int(c * APC), &full[d]);
        }
    }
    for (long long i = 0;; ++i) {
        const long long c = blockIdx.x + i * gridDim.x;
        if (c >= chunks) break;
        const int b = int(i % DEPTH);
        const uint32_t parity = uint32_t((i / DEPTH) & 1);
        unsigned char* buf = base + b * buf_bytes;
        // wait for the chunk, with a time limit agreed by the whole CTA
        bool ok = tma::mbar_try_wait(&full[b], parity);
        if (!ok) {
            const long long t0 = clock64();
            while (!(ok = tma::mbar_try_wait(&full[b], parity)) && clock64() - t0 < tma::kWaitLimit) {
            }
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicAdd(&status->timeouts, 1ull);
                tma::wait_group_all();
            }
            return;
        }
        // this thread's K elements: 16-byte chunks g = t*CH + q of its array
        const uint32_t row0 = uint32_t(slot * rows);
        R v[S::K];
        sfor<0, CH>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const int g = t * CH + q;
            if (g < valid_chunks) {
                const uint32_t row = row0 + uint32_t(g >> 3);
                const uint4 u = *reinterpret_cast<const uint4*>(buf + tma::swz(row, uint32_t(g & 7)));
                sfor<0, PER>([&](auto jc) {
                    constexpr int j = decltype(jc)::value;
                    M m;
                    from_u4<j>(u, m);
                    v[q * PER + j] = E::from_mem(m, g * PER + j);
                });
            } else {
                sfor<0, PER>([&](auto jc) { v[q * PER + decltype(jc)::value] = E::pad(); });
            }
        });
        R* no_smem = nullptr;
        network<E, S>(v, t, no_smem, no_smem);
        sfor<0, CH>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const int g = t * CH + q;
            if (g < valid_chunks) {
                const uint32_t row = row0 + uint32_t(g >> 3);
                uint4 u;
                sfor<0, PER>([&](auto jc) {
                    constexpr int j = decltype(jc)::value;
                    to_u4<j>(u, E::to_mem(v[q * PER + j]));
                });
                *reinterpret_cast<uint4*>(buf + tma::swz(row, uint32_t(g & 7))) = u;
            }
        });
        tma::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tma::store_3d(&tout, 0, 0, int(c * APC), buf);
            tma::commit_group();
            // refill the buffer stored one iteration ago with the chunk DEPTH-1 ahead
            const long long cn = c + (long long)(DEPTH - 1) * gridDim.x;
            if (cn < chunks) {
                const int nb = int((i + DEPTH - 1) % DEPTH);
                tma::wait_group_read<1>();
                tma::mbar_expect_tx(&full[nb], box_bytes);
                tma::load_3d(base + nb * buf_bytes, &tin, 0, 0, int(cn * APC), &full[nb]);
            }
        }
    }
    if (tid == 0) tma::wait_group_all();
}

}  // namespace b200s
