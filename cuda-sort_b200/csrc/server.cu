// The b200sort server: continuous batching of arriving sort requests on one
// GPU (the scheduling policy is in serving_core.hpp; this file is its CUDA
// backend and the C ABI).
//
// Device layout.  The server owns one arena of budget_bytes.  A batch is one
// contiguous arena region holding its requests back to back, each request's
// slot rounded up to 16 bytes and its tail filled with maximum-key padding,
// so that every array starts 16-byte aligned (whole 128-bit tile loads) and
// the ragged kernels see an ordinary CSR batch.  Padding that follows an
// array's valid elements never moves under the network's keep-own rule (and
// sorts after every valid element in the stable mode), so the first n
// elements of a slot are exactly the request sorted alone.
//
// A batch on slot s, all on stream s:
//   1. one host-to-device copy of the batch's offsets and request descriptors
//      (from this slot's pinned staging buffer),
//   2. host-memory requests: one cudaMemcpyAsync each into their arena slots,
//   3. k_stage (in): device-memory requests copied into their slots, padding
//      written, one CTA per 16 KB chunk of the batch,
//   4. the ragged sort of the region in place (a per-slot plan, direct
//      launches: the persistent length-bucketed kernel plus cluster kernels),
//   5. k_stage (out): device-memory results copied to their destinations,
//   6. host-memory requests: one cudaMemcpyAsync each back to the host,
//   7. an event the scheduler polls.
// A batch of at most kDirectMax requests instead launches the packed sort once
// per request, straight from its source to its destination.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "b200sort.h"
#include "serving_core.hpp"

namespace b200s {

b200s_status set_error(b200s_status s, const std::string& msg);
b200s_status cuda_error(cudaError_t e, const char* what);
size_t elem_bytes(int dtype);

namespace {

constexpr int kChunkBytes = 16384;
constexpr int kDirectMax = 3;  // batches of up to this many requests launch per request
constexpr int kStageThreads = 256;

struct Desc {
    const void* src;
    void* dst;
    long long arena_elem;
    int n;
    int n_pad;
    int chunk_begin;
    unsigned mem;
};

// Copy [b0, b1) bytes from s to d with 16-byte accesses when both are
// 16-byte aligned, else 4-byte words (every element type is a multiple of 4).
__device__ __forceinline__ void copy_span(char* d, const char* s, long long b0, long long b1) {
    if (b1 <= b0) return;
    long long i = b0;
    if (((reinterpret_cast<uintptr_t>(d + b0) | reinterpret_cast<uintptr_t>(s + b0)) & 15u) == 0) {
        const long long v1 = b0 + (b1 - b0) / 16 * 16;
        for (long long k = b0 + 16LL * threadIdx.x; k < v1; k += 16LL * blockDim.x)
            *reinterpret_cast<uint4*>(d + k) = *reinterpret_cast<const uint4*>(s + k);
        i = v1;
    }
    for (long long k = i + 4LL * threadIdx.x; k < b1; k += 4LL * blockDim.x)
        *reinterpret_cast<unsigned*>(d + k) = *reinterpret_cast<const unsigned*>(s + k);
}

// dir 0: stage requests into the arena and write padding; dir 1: copy the
// sorted valid prefixes out.  Host-memory requests move by cudaMemcpyAsync;
// here they only receive their padding.
__global__ void __launch_bounds__(kStageThreads) k_stage(const Desc* __restrict__ desc, int count, char* arena,
                                                         int eb, unsigned pad0, unsigned pad1, int dir) {
    int lo = 0, hi = count - 1;
    const int c = int(blockIdx.x);
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (desc[mid].chunk_begin <= c) lo = mid;
        else hi = mid - 1;
    }
    const Desc r = desc[lo];
    const long long valid = (long long)r.n * eb;
    const long long total = (long long)r.n_pad * eb;
    const long long b0 = (long long)(c - r.chunk_begin) * kChunkBytes;
    const long long b1 = b0 + kChunkBytes < total ? b0 + kChunkBytes : total;
    char* slot = arena + r.arena_elem * eb;
    const long long v1 = b1 < valid ? b1 : valid;
    if (dir == 0) {
        if (r.mem == B200S_MEM_DEVICE) copy_span(slot, static_cast<const char*>(r.src), b0, v1);
        // padding: whole words of the maximum-key element pattern
        for (long long k = (b0 > valid ? b0 : valid) + 4LL * threadIdx.x; k < b1; k += 4LL * blockDim.x)
            *reinterpret_cast<unsigned*>(slot + k) = ((k / 4) & 1) ? pad1 : pad0;
    } else if (r.mem == B200S_MEM_DEVICE) {
        copy_span(static_cast<char*>(r.dst), slot, b0, v1);
    }
}

class CudaBackend {
public:
    struct Slot {
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        b200s_plan* plan = nullptr;
        char* h_meta = nullptr;  // pinned: offsets, then descriptors
        char* d_meta = nullptr;
    };

    ~CudaBackend() { release(); }

    b200s_status init(const b200s_server_config& c, std::string* err) {
        device_ = c.device;
        dtype_ = c.dtype;
        flags_ = c.flags;
        eb_ = int(b200s::elem_bytes(c.dtype));
        align_ = 16 / eb_ > 0 ? 16 / eb_ : 1;
        max_batch_ = c.max_batch;
        max_len_ = b200s_ragged_max_length(c.dtype, c.flags);
        // padding element: maximum key (and maximum payload), as 2 words
        pad0_ = dtype_ == B200S_I32 || dtype_ == B200S_I32_I32 ? 0x7fffffffu : 0xffffffffu;
        pad1_ = dtype_ == B200S_I32_I32 ? 0x7fffffffu : pad0_;
        cudaError_t e = cudaSetDevice(device_);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice", err);
        const int64_t per = int64_t(align_) * eb_;
        arena_elems_ = c.budget_bytes / per * align_;
        if (arena_elems_ <= 0) {
            *err = "budget_bytes below one 16-byte slot";
            return B200S_ERR_INVALID_ARGUMENT;
        }
        e = cudaMalloc(&arena_, size_t(arena_elems_) * size_t(eb_));
        if (e != cudaSuccess) return cuda_fail(e, "server arena allocation", err);
        meta_bytes_ = offsets_bytes() + size_t(max_batch_) * sizeof(Desc);
        slots_.resize(size_t(c.max_inflight));
        for (Slot& s : slots_) {
            if ((e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "server stream", err);
            if ((e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "server event", err);
            if ((e = cudaMallocHost(&s.h_meta, meta_bytes_)) != cudaSuccess)
                return cuda_fail(e, "server pinned staging", err);
            if ((e = cudaMalloc(&s.d_meta, meta_bytes_)) != cudaSuccess)
                return cuda_fail(e, "server descriptor buffer", err);
            const b200s_status st = b200s_plan_create(&s.plan, b200s_dtype(dtype_), flags_ | B200S_PLAN_NO_GRAPH,
                                                      max_batch_, device_);
            if (st != B200S_OK) {
                *err = std::string("server plan: ") + b200s_last_error();
                return st;
            }
        }
        return B200S_OK;
    }

    int slots() const { return int(slots_.size()); }
    int64_t arena_elems() const { return arena_elems_; }
    int elem_bytes() const { return eb_; }
    int align_elems() const { return align_; }
    int32_t max_length() const { return max_len_; }

    b200s_status launch(int slot, const serving::Item* items, int count, int64_t region_elem,
                        int64_t region_elems, std::string* err) {
        Slot& s = slots_[size_t(slot)];
        cudaError_t e = cudaSetDevice(device_);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice", err);
        if (region_elems > INT_MAX) {
            *err = "batch region beyond int32 offsets";
            return B200S_ERR_INVALID_ARGUMENT;
        }
        if (count <= kDirectMax) return launch_direct(s, items, count, err);
        int32_t* off = reinterpret_cast<int32_t*>(s.h_meta);
        Desc* desc = reinterpret_cast<Desc*>(s.h_meta + offsets_bytes());
        int chunks = 0;
        bool any_device = false;
        for (int i = 0; i < count; ++i) {
            const serving::Item& it = items[i];
            off[i] = int32_t(it.arena_elem - region_elem);
            desc[i] = Desc{it.req->src, it.req->dst, (long long)it.arena_elem, it.req->n, it.n_pad, chunks,
                           it.req->mem};
            chunks += int((int64_t(it.n_pad) * eb_ + kChunkBytes - 1) / kChunkBytes);
            any_device = any_device || it.req->mem == B200S_MEM_DEVICE;
        }
        off[count] = int32_t(region_elems);
        const size_t obytes = offsets_bytes();
        // offsets and descriptors are one copy (descriptors start at obytes)
        e = cudaMemcpyAsync(s.d_meta, s.h_meta, obytes + size_t(count) * sizeof(Desc), cudaMemcpyHostToDevice,
                            s.stream);
        if (e != cudaSuccess) return cuda_fail(e, "server descriptor upload", err);
        char* arena = static_cast<char*>(arena_);
        for (int i = 0; i < count; ++i)
            if (items[i].req->mem == B200S_MEM_HOST) {
                e = cudaMemcpyAsync(arena + items[i].arena_elem * eb_, items[i].req->src,
                                    size_t(items[i].req->n) * size_t(eb_), cudaMemcpyHostToDevice, s.stream);
                if (e != cudaSuccess) return cuda_fail(e, "server host-to-device copy", err);
            }
        const Desc* d_desc = reinterpret_cast<const Desc*>(s.d_meta + obytes);
        k_stage<<<chunks, kStageThreads, 0, s.stream>>>(d_desc, count, arena, eb_, pad0_, pad1_, 0);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "stage-in launch", err);
        void* region = arena + region_elem * eb_;
        // the host copy of the offsets lets the plan skip the classes this batch has no array in
        const b200s_status st = b200s_sort_ragged_hinted(s.plan, region, region,
                                                         reinterpret_cast<const int32_t*>(s.d_meta), off, count,
                                                         s.stream);
        if (st != B200S_OK) {
            *err = std::string("server batch sort: ") + b200s_last_error();
            return st;
        }
        if (any_device) {
            k_stage<<<chunks, kStageThreads, 0, s.stream>>>(d_desc, count, arena, eb_, pad0_, pad1_, 1);
            if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "stage-out launch", err);
        }
        for (int i = 0; i < count; ++i)
            if (items[i].req->mem == B200S_MEM_HOST) {
                e = cudaMemcpyAsync(items[i].req->dst, arena + items[i].arena_elem * eb_,
                                    size_t(items[i].req->n) * size_t(eb_), cudaMemcpyDeviceToHost, s.stream);
                if (e != cudaSuccess) return cuda_fail(e, "server device-to-host copy", err);
            }
        if ((e = cudaEventRecord(s.done, s.stream)) != cudaSuccess) return cuda_fail(e, "server event record", err);
        return B200S_OK;
    }

    // A batch of a few requests skips staging and binning: each request is
    // one packed launch of one array, from its source into its destination
    // (host-memory requests through their arena slot).  At low load this is
    // the whole path; the result equals the batched path's (the network's
    // output does not depend on the working length or the padding).
    b200s_status launch_direct(Slot& s, const serving::Item* items, int count, std::string* err) {
        char* arena = static_cast<char*>(arena_);
        cudaError_t e;
        for (int i = 0; i < count; ++i) {
            const serving::Request& r = *items[i].req;
            const size_t bytes = size_t(r.n) * size_t(eb_);
            const void* in = r.src;
            void* out = r.dst;
            if (r.mem == B200S_MEM_HOST) {
                out = arena + items[i].arena_elem * eb_;
                in = out;
                if ((e = cudaMemcpyAsync(out, r.src, bytes, cudaMemcpyHostToDevice, s.stream)) != cudaSuccess)
                    return cuda_fail(e, "server host-to-device copy", err);
            }
            const b200s_status st =
                b200s_sort_packed(b200s_dtype(dtype_), in, out, r.n, 1, flags_, nullptr, s.stream);
            if (st != B200S_OK) {
                *err = std::string("server request sort: ") + b200s_last_error();
                return st;
            }
            if (r.mem == B200S_MEM_HOST &&
                (e = cudaMemcpyAsync(r.dst, out, bytes, cudaMemcpyDeviceToHost, s.stream)) != cudaSuccess)
                return cuda_fail(e, "server device-to-host copy", err);
        }
        if ((e = cudaEventRecord(s.done, s.stream)) != cudaSuccess) return cuda_fail(e, "server event record", err);
        return B200S_OK;
    }

    int query(int slot, std::string* err) {
        cudaSetDevice(device_);
        const cudaError_t e = cudaEventQuery(slots_[size_t(slot)].done);
        if (e == cudaSuccess) return 1;
        if (e == cudaErrorNotReady) return 0;
        *err = std::string("server batch: ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        return -1;
    }

private:
    size_t offsets_bytes() const { return ((size_t(max_batch_) + 1) * sizeof(int32_t) + 15) & ~size_t(15); }

    static b200s_status cuda_fail(cudaError_t e, const char* what, std::string* err) {
        *err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        return e == cudaErrorMemoryAllocation ? B200S_ERR_OUT_OF_MEMORY : B200S_ERR_CUDA;
    }

    void release() {
        cudaSetDevice(device_);
        for (Slot& s : slots_) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            if (s.plan) b200s_plan_destroy(s.plan);
            if (s.d_meta) cudaFree(s.d_meta);
            if (s.h_meta) cudaFreeHost(s.h_meta);
            if (s.done) cudaEventDestroy(s.done);
            if (s.stream) cudaStreamDestroy(s.stream);
        }
        slots_.clear();
        if (arena_) cudaFree(arena_);
        arena_ = nullptr;
    }

    int device_ = 0, dtype_ = 0, eb_ = 4, align_ = 4, max_batch_ = 0;
    uint32_t flags_ = 0;
    int32_t max_len_ = 0;
    unsigned pad0_ = 0, pad1_ = 0;
    void* arena_ = nullptr;
    int64_t arena_elems_ = 0;
    size_t meta_bytes_ = 0;
    std::vector<Slot> slots_;
};

}  // namespace
}  // namespace b200s

using namespace b200s;

struct b200s_server {
    std::unique_ptr<serving::ServerCore<CudaBackend>> core;
};

namespace {

b200s_status server_error(b200s_status s, const std::string& what) { return set_error(s, what); }

}  // namespace

extern "C" {

b200s_status b200s_server_create(b200s_server** out, const b200s_server_config* config) {
    if (!out || !config) return set_error(B200S_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    b200s_server_config c = *config;
    if (c.dtype < 0 || c.dtype > 3) return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (c.flags & ~(B200S_STABLE | B200S_SORTED_CHECK))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown flag bits");
    if (c.budget_bytes < 0 || c.max_inflight < 0 || c.max_batch < 0 || c.max_queue < 0)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "negative server limit");
    if (c.budget_bytes == 0) c.budget_bytes = int64_t(1) << 30;
    if (c.max_inflight == 0) c.max_inflight = 4;
    if (c.max_batch == 0) c.max_batch = 4096;
    if (c.max_queue == 0) c.max_queue = 65536;
    if (c.max_inflight > 64 || c.max_batch > (1 << 20) || c.max_queue > (int64_t(1) << 26))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "server limit out of range");
    auto be = std::make_unique<CudaBackend>();
    std::string err;
    const b200s_status st = be->init(c, &err);
    if (st != B200S_OK) return server_error(st, err);
    serving::Limits lim;
    lim.max_batch_arrays = c.max_batch;
    lim.max_queue = c.max_queue;
    lim.max_batch_elems = INT_MAX;
    auto* s = new b200s_server();
    s->core = std::make_unique<serving::ServerCore<CudaBackend>>(std::move(be), lim);
    *out = s;
    return B200S_OK;
}

b200s_status b200s_server_destroy(b200s_server* s) {
    if (!s) return B200S_OK;
    s->core->shutdown();
    delete s;  // the backend synchronises its streams and frees the arena
    return B200S_OK;
}

b200s_status b200s_server_submit(b200s_server* s, const void* src, void* dst, int32_t n, uint32_t mem,
                                 uint64_t* ticket) {
    if (!s) return set_error(B200S_ERR_INVALID_ARGUMENT, "null server");
    std::string err;
    const b200s_status st = s->core->submit(src, dst, n, mem, ticket, &err);
    return st == B200S_OK ? st : server_error(st, err);
}

b200s_status b200s_server_submit_arrived(b200s_server* s, const void* src, void* dst, int32_t n, uint32_t mem,
                                         int64_t arrival_ns, uint64_t* ticket) {
    if (!s) return set_error(B200S_ERR_INVALID_ARGUMENT, "null server");
    if (arrival_ns <= 0) return set_error(B200S_ERR_INVALID_ARGUMENT, "arrival time must be positive");
    std::string err;
    const b200s_status st = s->core->submit(src, dst, n, mem, ticket, &err, arrival_ns);
    return st == B200S_OK ? st : server_error(st, err);
}

int64_t b200s_server_clock_ns(void) { return serving::now_ns(); }

b200s_status b200s_server_wait(b200s_server* s, uint64_t ticket, int64_t timeout_us, b200s_status* result) {
    if (!s) return set_error(B200S_ERR_INVALID_ARGUMENT, "null server");
    std::string err;
    const b200s_status st = s->core->wait(ticket, timeout_us, result, &err);
    if (st == B200S_OK && result && *result == B200S_ERR_CUDA) set_error(B200S_ERR_CUDA, s->core->last_error());
    return st == B200S_OK ? st : server_error(st, err);
}

b200s_status b200s_server_poll(b200s_server* s, uint64_t ticket, int32_t* state, b200s_status* result) {
    if (!s || !state) return set_error(B200S_ERR_INVALID_ARGUMENT, "null argument");
    int status = B200S_OK;
    *state = s->core->state_of(ticket, &status);
    if (result) *result = b200s_status(status);
    return B200S_OK;
}

b200s_status b200s_server_cancel(b200s_server* s, uint64_t ticket) {
    if (!s) return set_error(B200S_ERR_INVALID_ARGUMENT, "null server");
    std::string err;
    const b200s_status st = s->core->cancel(ticket, &err);
    return st == B200S_OK ? st : server_error(st, err);
}

b200s_status b200s_server_drain(b200s_server* s, int64_t timeout_us) {
    if (!s) return set_error(B200S_ERR_INVALID_ARGUMENT, "null server");
    std::string err;
    const b200s_status st = s->core->drain(timeout_us, &err);
    return st == B200S_OK ? st : server_error(st, err);
}

b200s_status b200s_server_stats_get(b200s_server* s, b200s_server_stats* out, int32_t reset) {
    if (!s || !out) return set_error(B200S_ERR_INVALID_ARGUMENT, "null argument");
    s->core->stats(out, reset != 0);
    return B200S_OK;
}

}  // extern "C"
