/*
 * b200sort — batched small-array sort for NVIDIA B200 (sm_100a), C ABI.
 *
 * Drop-in for the one-CTA-per-array bitonic path of berenger-eu/cuda-sort.
 * The reference exposes that path as header-only CUDA templates launched one
 * CTA per array over a packed batch; this library exports the same operation
 * as plain C entry points over caller-owned device buffers:
 *
 *   reference                                              this library
 *   ---------------------------------------------------    ---------------------------
 *   cusort_v6::Sort<T,W,Threads,...>(in, out, n)           b200s_sort_packed
 *     cusort_v6.hpp:144-178, kernel cusort_v6.hpp:181-184
 *   batched wrapper benchmarkSortV6Register<<<A,...>>>      b200s_sort_packed
 *     (segment = data + blockIdx.x * n), bench.cu:389-393
 *   cusort_experiment::Sort / Sort_1Block_v4_xor /          b200s_sort_packed
 *     Sort_1Block_v5_static, cusort_experiments.hpp:366-419
 *   Sort_1Block_gt32_d_extsm_v3 (cusort.hpp:1229-1231),     b200s_sort_packed
 *     Sort_1Warp_SM_le32_d (cusort.hpp:574-575)
 *   SortPartitionsAdaptive_outofplace over CSR partitions   b200s_sort_ragged / b200s_plan_*
 *     (cusort.hpp:2309-2352; one launch, ragged lengths)
 *   Batch::run host-to-device restore + launch              b200s_sort_packed_host
 *     (bench.cu:320-352)
 *
 * Semantics shared with the reference:
 *   - ascending by key; records (IntAndData, intanddata.hpp:9-52) compare by
 *     key only and move with their payload;
 *   - the default (unstable) mode applies the reference's comparator network
 *     with its keep-own rule on ties, so record outputs, including the order
 *     of equal keys, are identical to the reference's;
 *   - in-place operation (d_in == d_out) is allowed, as bench.cu:392 uses it;
 *   - the caller owns every buffer; the sort entry points allocate nothing.
 * Differences: errors are returned as status codes instead of device asserts
 * or exit() (cusort.hpp:240-245); every call takes a stream; lengths are not
 * capped by the reference's 48 KB shared-memory rule (cusort.hpp:231-237).
 *
 * Streams are passed as `void*` holding a cudaStream_t (NULL = legacy default
 * stream).  Entry points are safe to call from several host threads as long
 * as each session/plan is used by one thread at a time.
 */
#ifndef B200SORT_H
#define B200SORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum b200s_status {
    B200S_OK = 0,
    B200S_ERR_INVALID_ARGUMENT = 1, /* null pointer, negative size, bad flag */
    B200S_ERR_UNSUPPORTED = 2,      /* no compiled kernel covers this dtype/length/tile */
    B200S_ERR_CUDA = 3,             /* a CUDA runtime call failed; see b200s_last_error() */
    B200S_ERR_OUT_OF_MEMORY = 4,    /* a session/plan/server could not allocate */
    B200S_ERR_TIMEOUT = 5,          /* a bounded wait gave up */
    B200S_ERR_BUDGET = 6,           /* request larger than the server's device-memory budget */
    B200S_ERR_BUSY = 7,             /* the server's request table is full; retry later */
    B200S_ERR_CANCELLED = 8         /* result of a request cancelled before it was admitted */
} b200s_status;

typedef enum b200s_dtype {
    B200S_I32 = 0,     /* int32_t keys                                              */
    B200S_I32_I32 = 1, /* {int32_t key; int32_t data;}  == IntAndData, 8 bytes      */
    B200S_U64 = 2,     /* uint64_t keys                                             */
    B200S_U64_I32 = 3  /* {uint64_t key; int32_t data; int32_t reserved;}, 16 bytes */
} b200s_dtype;

/* flags */
#define B200S_STABLE 1u       /* ties keep input order (bit-exact std::stable_sort) */
#define B200S_SORTED_CHECK 2u /* the reference's `Sorted` switch (cusort_v6.hpp:103-128): the
                                 packed path tests each array before sorting and skips the
                                 network when it is already in order (in place: the store
                                 too); the transposed-network form also tests after every
                                 stage of span >= 16.  The output is identical either way.
                                 The TMA form runs form 0 instead; the cluster and ragged
                                 paths accept the flag and sort in full. */
#define B200S_PLAN_NO_GRAPH 0x100u /* plan flag: launch the ragged sequence directly
                                      instead of replaying a captured CUDA graph */

/* A tile shape: how one array is laid over threads.  K = 2^log2_items
 * elements per thread, 2^log2_lanes lanes per array inside a warp,
 * 2^log2_warps warps per CTA-slice of the array and 2^log2_ctas CTAs (a
 * thread-block cluster) per array.  The working length is
 * W = 2^(log2_items + log2_lanes + log2_warps + log2_ctas) and must be >= n. */
typedef struct b200s_tile {
    int32_t log2_items;
    int32_t log2_lanes;
    int32_t log2_warps;
    int32_t cta_threads; /* threads per CTA (output of the query functions) */
    int32_t persistent;  /* launch form. 0: one launch slot per array group; 1: grid sized
                            to the resident capacity, each group prefetching its next array
                            into registers; 2: persistent CTAs streaming chunks of arrays
                            through shared memory with TMA loads and stores (used when every
                            array is whole 128-byte rows, at most 256, and the buffers are
                            16-byte aligned; form 0 otherwise); 3: transposed network, every
                            comparator layer in registers with the tile re-laid out through
                            shared memory between register windows (single-warp tiles of
                            int32 and uint64 keys, IntAndData records and stable records up
                            to W = 1024, with element-aligned buffers; and the multi-warp
                            and cluster tiles of every element type; b200s_tile_info's
                            xpose_form tells which; form 0 otherwise) */
    int32_t log2_ctas;   /* CTAs per array: 0 for single-CTA tiles (cluster tiles of one
                            CTA exist only where no single-CTA tile of that shape does) */
} b200s_tile;

const char* b200s_version(void);
const char* b200s_status_string(b200s_status status);
/* Message of the last failing call on this host thread ("" if none). */
const char* b200s_last_error(void);

/* Largest array length the packed path handles for dtype/flags. */
int32_t b200s_max_length(b200s_dtype dtype, uint32_t flags);

/* Compiled tiles, for autotuning: index in [0, b200s_tile_count). */
int32_t b200s_tile_count(b200s_dtype dtype, uint32_t flags);
b200s_status b200s_tile_get(b200s_dtype dtype, uint32_t flags, int32_t index, b200s_tile* out);
/* Tile the library uses for arrays of length n when the caller passes none. */
b200s_status b200s_default_tile(b200s_dtype dtype, uint32_t flags, int32_t n, b200s_tile* out);
/* Resources of the kernel that sorts arrays of length n with `tile` (NULL:
 * the default tile), as the reference's bench reports them for its kernels
 * (bench.cu:425-440): registers and local memory per thread, shared memory
 * per CTA, threads per CTA, and CTAs resident per SM (computed from those). */
typedef struct b200s_tile_info {
    int32_t registers_per_thread;
    int32_t local_bytes_per_thread;
    int32_t shared_bytes;
    int32_t cta_threads;
    int32_t active_ctas_per_sm;
    int32_t working;        /* working length W of the tile */
    int32_t arrays_per_cta; /* 0 for cluster tiles (several CTAs per array) */
    int32_t tma_form;       /* 1 if launch form 2 runs a TMA kernel for this tile and n */
    int32_t xpose_form;     /* 1 if launch form 3 runs a transposed-network kernel for this tile */
} b200s_tile_info;
b200s_status b200s_tile_info_get(b200s_dtype dtype, uint32_t flags, const b200s_tile* tile, int32_t n,
                                 b200s_tile_info* out);
/* CTAs of the TMA-pipelined kernels on the current device that stopped
 * waiting for a load after about a second (each left its chunk unsorted).
 * Always 0 unless the device misbehaves; a cumulative count. */
b200s_status b200s_tma_timeouts(int64_t* count);
/* Test hook for failure detection: while enabled, every TMA-pipelined launch
 * on the current device expects 16 bytes more per chunk than its loads
 * deliver, so its bounded wait runs out (about a second per CTA), each CTA
 * counts itself in b200s_tma_timeouts and returns with its chunks unsorted;
 * nothing faults.  Disable before any real work. */
b200s_status b200s_test_stall_tma_loads(int32_t enable);
/* Replace rows of the default tile table from a CSV file; '#' starts a
 * comment.  Packed rows: dtype,flags,log2_w,log2_items,log2_lanes,log2_warps
 * [,form[,log2_ctas]] (form: 0 .. 3 as b200s_tile.persistent; log2_ctas: CTAs
 * per array of a cluster tile, default 0).  Ragged rows: r,dtype,flags,log2_w,family
 * [,log2_items,log2_lanes,log2_warps,form] (0: the persistent kernel with the larger per-thread tile, 1: with
 * the smaller one, 2: a launch of its own, in the single-CTA tile and form (0 or 3) given, or without them the
 * packed table's tile and form for that length), read by plans created afterwards.
 * Returns the number of rows applied in *applied. */
b200s_status b200s_load_tile_table(const char* path, int32_t* applied);

/* Sort `arrays` independent arrays of n elements each, packed back to back
 * (array a at element offset a*n), from d_in into d_out (device pointers; may
 * be equal).  tile == NULL uses the default tile for n.  The single-CTA
 * launches allow programmatic stream serialization: their CTAs may be
 * scheduled while the stream's previous kernel drains, and each waits for
 * that kernel's completion (griddepcontrol.wait) before touching memory, so
 * stream order is kept for any producer. */
b200s_status b200s_sort_packed(b200s_dtype dtype, const void* d_in, void* d_out, int32_t n,
                               int64_t arrays, uint32_t flags, const b200s_tile* tile,
                               void* stream);

/* ---- ragged batches (CSR offsets) ----------------------------------------
 * Array a occupies elements [offsets[a], offsets[a+1]) of the flat buffer
 * (int32 offsets, arrays + 1 entries, non-decreasing).  A plan owns the
 * scratch of the bucketed launch (a control block and 2 * max_arrays ids)
 * and, unless B200S_PLAN_NO_GRAPH is set, a CUDA graph of the launch
 * sequence, re-captured when the buffers or the array count change.  Replaces
 * the reference's partition sort over CSR partitions
 * (SortPartitionsAdaptive_outofplace, cusort.hpp:2309-2352). */
typedef struct b200s_plan b200s_plan;
b200s_status b200s_plan_create(b200s_plan** out, b200s_dtype dtype, uint32_t flags, int64_t max_arrays,
                               int32_t device);
b200s_status b200s_plan_destroy(b200s_plan* plan);
/* Longest array the ragged path sorts; longer arrays are counted, not sorted. */
int32_t b200s_ragged_max_length(b200s_dtype dtype, uint32_t flags);
/* The plan's launch sequence: binning, then the persistent length-bucketed
 * kernel on `stream`, with the length classes that the tile table gives a
 * launch of their own and the cluster classes above the persistent kernel's
 * range on side streams, joined before return (graph-replayed unless
 * B200S_PLAN_NO_GRAPH). */
b200s_status b200s_sort_ragged(b200s_plan* plan, const void* d_in, void* d_out, const int32_t* d_offsets,
                               int64_t arrays, void* stream);
/* b200s_sort_ragged for a caller that also holds the offsets on the host
 * (h_offsets: the same arrays + 1 values as d_offsets, read during the call).
 * A B200S_PLAN_NO_GRAPH plan then issues only the launches of the length
 * classes the batch holds: a launch of its own or a cluster class that no
 * array falls in is skipped, and so is the persistent kernel when every
 * array is in such a class.  Results equal b200s_sort_ragged's.  A graph plan
 * (or h_offsets == NULL) runs b200s_sort_ragged. */
b200s_status b200s_sort_ragged_hinted(b200s_plan* plan, const void* d_in, void* d_out, const int32_t* d_offsets,
                                      const int32_t* h_offsets, int64_t arrays, void* stream);
/* Arrays of the last b200s_sort_ragged that exceeded b200s_ragged_max_length
 * (synchronises `stream`). */
b200s_status b200s_plan_too_long(b200s_plan* plan, void* stream, int64_t* count);
/* Plain per-length form, for comparison: prepare groups the arrays by exact
 * length on the host (from host offsets) and uploads the id lists; each sort
 * then issues one launch per distinct length. */
b200s_status b200s_plan_prepare_plain(b200s_plan* plan, const int32_t* h_offsets, int64_t arrays);
/* The same grouped by power-of-two working length instead of exact length:
 * one launch per length class (W/2, W] with the tile of W, about log2 of the
 * longest array launches; a plain comparator without the launch count of the
 * per-length form.  b200s_sort_ragged_plain then runs these groups. */
b200s_status b200s_plan_prepare_plain_buckets(b200s_plan* plan, const int32_t* h_offsets, int64_t arrays);
b200s_status b200s_sort_ragged_plain(b200s_plan* plan, const void* d_in, void* d_out,
                                     const int32_t* d_offsets, void* stream);
int32_t b200s_plan_plain_launches(const b200s_plan* plan);

/* The leaf of the reference's partitioned large-array sort: replaces the
 * launch of SortPartitionsAdaptive_outofplace (cusort.hpp:2309-2352, launched
 * by HybridSortPartitionedV3 at cusort.hpp:2616-2628).  Sorts every partition
 * [d_counters[p], d_counters[p+1]) of d_in into the same range of d_out (out
 * of place; d_in == d_out is allowed), p < nb_parts, int32 CSR counters on
 * the device (nb_parts + 1 entries).  d_uniform (nb_parts device flags, may
 * be NULL) marks partitions that hold a single key value, which the
 * reference copies; sorting such a partition leaves it unchanged, so they go
 * through the same launch.  Unlike the reference's kernel, partitions up to
 * b200s_ragged_max_length are sorted (the reference sends those above its
 * 48 KB rule to a separate merge sort); longer ones are not written to d_out,
 * and the caller sorts them as the reference's merge path does.
 * Backed by a ragged plan cached per device, element type and stream (one
 * allocation the first time, re-captured graph when the buffers change);
 * b200s_release_partition_plans frees the cached plans. */
b200s_status b200s_sort_partitions(b200s_dtype dtype, uint32_t flags, const void* d_in, void* d_out,
                                   const int32_t* d_counters, const int32_t* d_uniform, int32_t nb_parts,
                                   void* stream);
b200s_status b200s_release_partition_plans(void);

/* No counterpart in the reference.  The ragged sort of b200s_sort_ragged for
 * callers that cannot allocate device memory: plugins inside a framework that
 * owns all device memory through its own pool, and latency-critical loops
 * where cudaMalloc's implicit device-wide synchronisation would stall other
 * work.  Instead of a plan's allocation it uses one fixed scratch array
 * compiled into the library (about 640 KiB on every GPU that loads the
 * library, held until the process exits), so:
 *   - at most B200S_NOALLOC_MAX_ARRAYS arrays per call; more is rejected
 *     with B200S_ERR_INVALID_ARGUMENT;
 *   - arrays longer than b200s_ragged_max_length(dtype, flags) are left
 *     unsorted (there is no plan to report them);
 *   - every call shares that scratch: calls whose work overlaps on the GPU
 *     (different streams, different host threads) race and corrupt each
 *     other; order them on one stream;
 *   - the first call on each device looks up the scratch's device address and
 *     sets kernel attributes; make that first call before any stream capture;
 *   - that address is kept for the life of the process: after a
 *     cudaDeviceReset of a device this entry point must not be called on it
 *     again (the reset reloads the library's device code elsewhere).
 * It runs the same kernels as b200s_sort_ragged (including the same cluster
 * tile for arrays above the persistent kernel's range) and calls no
 * cudaMalloc or cudaFree. */
#define B200S_NOALLOC_MAX_ARRAYS 32768
b200s_status b200s_sort_ragged_noalloc(b200s_dtype dtype, uint32_t flags, const void* d_in, void* d_out,
                                       const int32_t* d_offsets, int64_t arrays, void* stream);

/* ---- host-buffer entry point (end to end) ------------------------------- */
typedef struct b200s_session b200s_session;
b200s_status b200s_session_create(b200s_session** out, int32_t device);
b200s_status b200s_session_destroy(b200s_session* session);
/* Same as b200s_sort_packed, on host buffers: the batch is copied to the
 * device in chunks of whole arrays (a quarter of the batch, 2 to 64 MB), each
 * chunk sorted after its copy on one stream and copied back on another, so
 * that the copy back of one chunk overlaps the copy in of the next.  Pinned
 * host buffers give full PCIe bandwidth.  Returns after the output is in
 * h_out. */
b200s_status b200s_sort_packed_host(b200s_session* session, b200s_dtype dtype, const void* h_in,
                                    void* h_out, int32_t n, int64_t arrays, uint32_t flags);

/* ---- serving: continuous batching of arriving sort requests ---------------
 * No counterpart in the reference (it sorts batches it builds itself).  A
 * server owns a device arena of budget_bytes and a worker thread.  Requests
 * (one array each, of any length up to b200s_ragged_max_length) are queued by
 * b200s_server_submit from any host thread and return at once; the worker
 * admits queued requests into the next batch whenever one of max_inflight
 * device slots is free and the arena has room for them, stages them into the
 * arena, sorts the batch with the ragged kernels, and copies each result to
 * its destination.  Batches of different slots run on different streams and
 * overlap on the device; requests that arrive meanwhile wait in the queue and
 * form the next batch.  A request's result is identical to sorting it alone
 * (b200s_sort_packed with arrays = 1).  Sources and destinations stay valid
 * until the request finishes: B200S_MEM_DEVICE pointers are device memory (or
 * mapped pinned host memory) read and written by kernels; B200S_MEM_HOST
 * pointers are host memory copied with cudaMemcpyAsync (pinned is faster). */
#define B200S_MEM_DEVICE 0u
#define B200S_MEM_HOST 1u

/* request states (b200s_server_poll) */
#define B200S_REQ_FREE 0      /* unknown ticket, or its table entry was reused */
#define B200S_REQ_QUEUED 1
#define B200S_REQ_RUNNING 2
#define B200S_REQ_DONE 3
#define B200S_REQ_FAILED 4
#define B200S_REQ_CANCELLED 5

typedef struct b200s_server_config {
    int32_t device;
    b200s_dtype dtype;
    uint32_t flags;           /* B200S_STABLE */
    int64_t budget_bytes;     /* device arena for admitted requests (default 1 GiB when 0) */
    int32_t max_inflight;     /* batches on the device at once (default 4) */
    int32_t max_batch;        /* requests per batch (default 4096) */
    int64_t max_queue;        /* request table entries (default 65536) */
} b200s_server_config;

typedef struct b200s_server_stats {
    int64_t submitted, completed, failed, cancelled, rejected;
    int64_t batches, keys_completed, queued, inflight_batches;
    int64_t peak_arena_bytes, arena_bytes, max_batch_requests;
    double mean_batch_requests;
    double p50_us, p99_us, p999_us, max_us, mean_us; /* submit -> result written */
    double span_s;            /* first submit -> last completion */
} b200s_server_stats;

typedef struct b200s_server b200s_server;
b200s_status b200s_server_create(b200s_server** out, const b200s_server_config* config);
/* Cancels queued requests, waits for admitted ones, frees the arena. */
b200s_status b200s_server_destroy(b200s_server* server);
/* Queue one request of n elements; *ticket identifies it.  B200S_ERR_BUDGET
 * when it can never fit the arena, B200S_ERR_BUSY when max_queue requests are
 * pending, B200S_ERR_UNSUPPORTED beyond the longest sortable array. */
b200s_status b200s_server_submit(b200s_server* server, const void* src, void* dst, int32_t n, uint32_t mem,
                                 uint64_t* ticket);
/* Same, for a request that arrived at arrival_ns (b200s_server_clock_ns
 * timeline) before this call: its latency counts from then. */
b200s_status b200s_server_submit_arrived(b200s_server* server, const void* src, void* dst, int32_t n,
                                         uint32_t mem, int64_t arrival_ns, uint64_t* ticket);
/* The server's clock (monotonic nanoseconds). */
int64_t b200s_server_clock_ns(void);
/* Wait for a request (timeout_us < 0: no limit); *result is its outcome
 * (B200S_OK, B200S_ERR_CUDA, B200S_ERR_CANCELLED). */
b200s_status b200s_server_wait(b200s_server* server, uint64_t ticket, int64_t timeout_us, b200s_status* result);
b200s_status b200s_server_poll(b200s_server* server, uint64_t ticket, int32_t* state, b200s_status* result);
/* Cancel a request that has not been admitted yet. */
b200s_status b200s_server_cancel(b200s_server* server, uint64_t ticket);
/* Wait until no request is queued or running. */
b200s_status b200s_server_drain(b200s_server* server, int64_t timeout_us);
/* Counters and latency percentiles since creation or the last reset. */
b200s_status b200s_server_stats_get(b200s_server* server, b200s_server_stats* out, int32_t reset);

#ifdef __cplusplus
}
#endif

#endif /* B200SORT_H */
