// CUB BlockMergeSort baseline (NOT part of the product; built into its own
// library, libb200sort_cub.so, and only timed beside the product).
//
// Also Thrust's per-segment loop (one thrust::sort call per array, as the
// reference's thrust_segment_loop method times it, bench.cu:575-585).
//
// One CTA per array of a packed batch, in place: BlockLoad (warp transpose,
// maximum-key default) -> BlockMergeSort(valid_items, maximum) -> BlockStore,
// the library's standard block-sort sequence, as the reference times it
// (bench.cu:406-423).  For records, padding (payload INT_MAX) orders after a
// valid record with an equal key, so valid INT_MAX keys stay in the prefix.
#include <cub/block/block_load.cuh>
#include <cub/block/block_merge_sort.cuh>
#include <cub/block/block_store.cuh>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/sort.h>

#include <climits>
#include <cstdint>

namespace {

struct Rec {
    int key;
    int data;
};

struct LessI32 {
    __device__ bool operator()(const int& a, const int& b) const { return a < b; }
};
struct KeyLessRec {
    __host__ __device__ bool operator()(const Rec& a, const Rec& b) const { return a.key < b.key; }
};
struct LessRec {
    __device__ bool operator()(const Rec& a, const Rec& b) const {
        if (a.key == b.key) return a.data != INT_MAX && b.data == INT_MAX;
        return a.key < b.key;
    }
};

template <class T> __device__ T pad_value();
template <> __device__ int pad_value<int>() { return INT_MAX; }
template <> __device__ Rec pad_value<Rec>() { return Rec{INT_MAX, INT_MAX}; }

template <class T, class Less, int Threads, int Items>
__global__ void __launch_bounds__(Threads) cub_sort(T* data, int n) {
    using Load = cub::BlockLoad<T, Threads, Items, cub::BLOCK_LOAD_WARP_TRANSPOSE>;
    using Store = cub::BlockStore<T, Threads, Items, cub::BLOCK_STORE_WARP_TRANSPOSE>;
    using Sort = cub::BlockMergeSort<T, Threads, Items>;
    __shared__ union {
        typename Load::TempStorage load;
        typename Store::TempStorage store;
        typename Sort::TempStorage sort;
    } temp;
    T keys[Items];
    T* seg = data + size_t(blockIdx.x) * n;
    Load(temp.load).Load(seg, keys, n, pad_value<T>());
    __syncthreads();
    Sort(temp.sort).Sort(keys, Less{}, n, pad_value<T>());
    __syncthreads();
    Store(temp.store).Store(seg, keys, n);
}

template <class T, class Less, int Threads, int Items>
int launch(void* d, int n, int arrays, cudaStream_t st) {
    cub_sort<T, Less, Threads, Items><<<arrays, Threads, 0, st>>>(static_cast<T*>(d), n);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

template <class T, class Less, int W, int Threads>
int by_threads(int threads, void* d, int n, int arrays, cudaStream_t st) {
    if constexpr (Threads <= 1024) {
        if constexpr (Threads <= W && W / Threads <= 32) {
            if (threads == Threads) return launch<T, Less, Threads, W / Threads>(d, n, arrays, st);
        }
        return by_threads<T, Less, W, Threads * 2>(threads, d, n, arrays, st);
    }
    return 1;
}

template <class T, class Less, int W>
int by_working(int working, int threads, void* d, int n, int arrays, cudaStream_t st) {
    if constexpr (W <= 4096) {
        if (working == W) return by_threads<T, Less, W, 32>(threads, d, n, arrays, st);
        return by_working<T, Less, W * 2>(working, threads, d, n, arrays, st);
    }
    return 1;
}

}  // namespace

extern "C" {
// dtype 0: int32 keys, 1: {int32 key, int32 data}.  working = power of two
// >= max(32, n); threads a power of two with working/threads <= 32.
// Returns 0 ok, 1 configuration not compiled, 2 CUDA launch error.
int cub_block_merge_sort(int dtype, void* d, int n, int arrays, int working, int threads, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dtype == 0) return by_working<int, LessI32, 32>(working, threads, d, n, arrays, st);
    if (dtype == 1) return by_working<Rec, LessRec, 32>(working, threads, d, n, arrays, st);
    return 1;
}

// One thrust::sort per array on `stream`, in place (records by key only).
int thrust_segment_sort(int dtype, void* d, int n, int arrays, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (int a = 0; a < arrays; ++a) {
        if (dtype == 0) {
            int* p = static_cast<int*>(d) + size_t(a) * n;
            thrust::sort(thrust::cuda::par.on(st), p, p + n);
        } else if (dtype == 1) {
            Rec* p = static_cast<Rec*>(d) + size_t(a) * n;
            thrust::sort(thrust::cuda::par.on(st), p, p + n, KeyLessRec{});
        } else {
            return 1;
        }
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
}
