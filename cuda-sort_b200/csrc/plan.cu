// Ragged-batch plans: scratch, the persistent bucketed launch, its CUDA
// graph, and the plain per-length launches it is compared with.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "b200sort.h"
#define B200S_DEFINE_BIN_KERNELS
#include "ragged.cuh"
#include "registry.h"

namespace b200s {

b200s_status set_error(b200s_status s, const std::string& msg);
b200s_status cuda_error(cudaError_t e, const char* what);
int effective_stable(int dtype, uint32_t flags);
int ceil_log2(long long n);
int lookup_default_entry(int dtype, int stable, long long n, int* persistent);
b200s_status launch_packed(int idx, int persistent, const void* in, void* out, int n, long long arrays,
                           cudaStream_t st, unsigned opts = 0);

const std::vector<RaggedEntry>& ragged_registry() {
    static std::vector<RaggedEntry> all = [] {
        std::vector<RaggedEntry> v;
        register_ragged_i32(v);
        register_ragged_rec(v);
        register_ragged_u64(v);
        return v;
    }();
    return all;
}

namespace {

std::mutex g_mask_mutex;
unsigned g_family_mask[4][2] = {};
unsigned g_dedicated_mask[4][2] = {};
// the tile of a length class's own launch when its table row names one
// (registry index + 1; 0: the packed table's tile), and its launch form
int g_own_entry1[4][2][kMaxBuckets] = {};
int g_own_form[4][2][kMaxBuckets] = {};

const RaggedEntry* find_ragged(int dtype, int stable) {
    for (const RaggedEntry& e : ragged_registry())
        if (e.dtype == dtype && e.stable == stable) return &e;
    return nullptr;
}

}  // namespace

// Ragged table rows: family 0 (A) or 1 (B) runs the bucket in the persistent
// kernel with that shape family; family 2 gives the bucket its own launch of
// the packed tile the tile table chooses for its working length.
void set_ragged_family(int dtype, int stable, int log2w, int family, int own_entry, int own_form) {
    std::lock_guard<std::mutex> lock(g_mask_mutex);
    const int b = log2w - kRaggedLmin;
    if (b < 0 || b >= kMaxBuckets) return;
    g_own_entry1[dtype][stable][b] = family == 2 && own_entry >= 0 ? own_entry + 1 : 0;
    g_own_form[dtype][stable][b] = own_form;
    if (family == 1) g_family_mask[dtype][stable] |= 1u << b;
    else g_family_mask[dtype][stable] &= ~(1u << b);
    if (family == 2) g_dedicated_mask[dtype][stable] |= 1u << b;
    else g_dedicated_mask[dtype][stable] &= ~(1u << b);
}

unsigned ragged_family_mask(int dtype, int stable) {
    std::lock_guard<std::mutex> lock(g_mask_mutex);
    return g_family_mask[dtype][stable];
}

unsigned ragged_dedicated_mask(int dtype, int stable) {
    std::lock_guard<std::mutex> lock(g_mask_mutex);
    return g_dedicated_mask[dtype][stable];
}

// Registry entries of the dedicated buckets (bit b of `mask`: bucket b, W =
// 2^(kRaggedLmin + b)): the tabled single-CTA tile of that working length.
// Buckets without one (none tabled, or a cluster tile) stay in the persistent
// kernel: their bit is cleared in *mask.  idx[b] receives the entry.
// xc[b] (optional): the table's launch form for that length is 3 and the
// tile has the transposed-network form.
void dedicated_entries(int dtype, int stable, int nb, unsigned* mask, int* idx, bool* xc) {
    for (int b = 0; b < nb; ++b) {
        idx[b] = -1;
        if (xc) xc[b] = false;
        if (!((*mask >> b) & 1u)) continue;
        int persistent = 0;
        int e;
        {
            std::lock_guard<std::mutex> lock(g_mask_mutex);
            e = g_own_entry1[dtype][stable][b] - 1;
            persistent = g_own_form[dtype][stable][b];
        }
        if (e < 0) e = lookup_default_entry(dtype, stable, 1LL << (kRaggedLmin + b), &persistent);
        const KernelEntry* k = e >= 0 ? &registry()[size_t(e)] : nullptr;
        // a single-CTA tile with its blocked id-list launch, or (a cluster of
        // one CTA included) its transposed one when the table picks form 3
        const bool blocked = k && k->lc < 0 && k->launch_list_dev;
        const bool xform = k && k->lc <= 0 && persistent == 3 && k->launch_list_dev_xc;
        if (k && k->log2w == kRaggedLmin + b && (blocked || xform)) {
            idx[b] = e;
            if (xc) xc[b] = xform;
            else if (!blocked) {  // a caller that does not take the form: no launch it can run
                idx[b] = -1;
                *mask &= ~(1u << b);
            }
        } else {
            *mask &= ~(1u << b);
        }
    }
}

// Whether the cluster tile `entry` runs its transposed-network form: the
// table's launch form for its working length is 3 and the form is compiled.
bool cluster_xc(int dtype, int stable, int entry) {
    const KernelEntry& k = registry()[size_t(entry)];
    if (!k.launch_cluster_list_xc) return false;
    int form = 0;
    return lookup_default_entry(dtype, stable, 1LL << k.log2w, &form) >= 0 && form == 3;
}

}  // namespace b200s

using namespace b200s;

struct b200s_plan {
    int device = 0;
    int dtype = 0;
    int stable = 0;
    uint32_t flags = 0;
    long long max_arrays = 0;
    const RaggedEntry* rk = nullptr;
    unsigned family_mask = 0;
    unsigned dedicated_mask = 0;         // buckets with their own launch
    int dedicated_entry[kMaxBuckets] = {};
    bool dedicated_xc[kMaxBuckets] = {};  // run the tile's transposed-network form
    int grid = 0;       // persistent CTAs
    int bin_grid = 0;   // CTAs of the binning kernels
    void* scratch = nullptr;
    RaggedCtl* ctl = nullptr;
    int* ids = nullptr;
    int* oids = nullptr;          // cluster-bucket id lists, stride max_arrays
    BinSpec spec = {};
    int over_entry[kMaxOverflow] = {};  // registry index of each cluster bucket
    bool over_xc[kMaxOverflow] = {};
    static constexpr int kSides = 4;
    cudaStream_t capture = nullptr;
    cudaStream_t side[kSides] = {};  // cluster and dedicated buckets run beside the persistent kernel
    cudaEvent_t fork = nullptr, join[kSides] = {};
    // the graph of the last (in, out, offsets, arrays)
    cudaGraphExec_t exec = nullptr;
    const void* g_in = nullptr;
    void* g_out = nullptr;
    const int* g_off = nullptr;
    long long g_arrays = -1;
    // plain per-length launches: ids grouped by exact length on the host
    int* plain_ids = nullptr;
    struct Group {
        int n, first, count, entry, persistent;
    };
    std::vector<Group> groups;
};

namespace {

// present / over_present: bit b set when bucket b (cluster class i) may hold
// an array; classes with a launch of their own are skipped when their bit is
// clear (all ones: launch everything, as a graph must).
b200s_status record_sequence(b200s_plan* p, const void* in, void* out, const int* off, int arrays,
                             cudaStream_t st, uint32_t present = ~0u, uint32_t over_present = ~0u) {
    cudaError_t e = cudaMemsetAsync(p->ctl, 0, sizeof(RaggedCtl), st);
    if (e != cudaSuccess) return cuda_error(e, "ragged control reset");
    const int bin_threads = 256;
    const int bin_grid = std::max(1, std::min(p->bin_grid, (arrays + bin_threads - 1) / bin_threads));
    k_bin_count<<<bin_grid, bin_threads, 0, st>>>(off, arrays, p->ctl, p->spec);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "bin count launch");
    k_bin_scatter<<<bin_grid, bin_threads, 0, st>>>(off, arrays, p->ctl, p->ids, p->oids, p->spec);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "bin scatter launch");
    // Fork: the cluster buckets and the dedicated buckets run on side streams
    // (largest first, round robin) while the persistent kernel runs on st;
    // join before returning.
    const int max_count = int(std::min<long long>(arrays, p->max_arrays));
    int used = 0;
    auto side_stream = [&](int k) -> cudaStream_t {
        const int s = k % b200s_plan::kSides;
        if (s >= used) {
            if (used == 0 && (e = cudaEventRecord(p->fork, st)) != cudaSuccess) return nullptr;
            if ((e = cudaStreamWaitEvent(p->side[s], p->fork, 0)) != cudaSuccess) return nullptr;
            used = s + 1;
        }
        return p->side[s];
    };
    int k = 0;
    for (int i = p->spec.n_over - 1; i >= 0; --i) {
        if (!((over_present >> i) & 1u)) continue;
        const KernelEntry& ke = registry()[size_t(p->over_entry[i])];
        cudaStream_t ss = side_stream(k++);
        if (!ss) return cuda_error(e, "fork");
        e = (p->over_xc[i] ? ke.launch_cluster_list_xc : ke.launch_cluster_list)(
            in, out, off, p->oids + size_t(i) * p->spec.stride, &p->ctl->ocount[i], max_count, ss);
        if (e != cudaSuccess) return cuda_error(e, "cluster bucket launch");
    }
    for (int b = p->spec.nb - 1; b >= 0; --b) {
        if (!((p->dedicated_mask >> b) & (present >> b) & 1u)) continue;
        const KernelEntry& ke = registry()[size_t(p->dedicated_entry[b])];
        cudaStream_t ss = side_stream(k++);
        if (!ss) return cuda_error(e, "fork");
        e = (p->dedicated_xc[b] ? ke.launch_list_dev_xc : ke.launch_list_dev)(
            in, out, off, p->ids, &p->ctl->count[b], &p->ctl->base[b], &p->ctl->dhead[b], max_count, ss);
        if (e != cudaSuccess) return cuda_error(e, "dedicated bucket launch");
    }
    const uint32_t all = (1u << p->spec.nb) - 1u;
    if (present & all & ~p->dedicated_mask) {
        e = p->rk->launch(in, out, off, p->ids, p->ctl, p->family_mask, p->dedicated_mask, p->grid, st);
        if (e != cudaSuccess) return cuda_error(e, "ragged sort launch");
    }
    for (int s = 0; s < used; ++s) {
        if ((e = cudaEventRecord(p->join[s], p->side[s])) != cudaSuccess) return cuda_error(e, "join record");
        if ((e = cudaStreamWaitEvent(st, p->join[s], 0)) != cudaSuccess) return cuda_error(e, "join wait");
    }
    return B200S_OK;
}

}  // namespace

namespace b200s {

// Cluster kernels that extend the persistent kernel's range: consecutive
// working lengths above its largest bucket, each the cluster tile with the
// fewest CTAs per array (the throughput tile).  Returns the number found.
int overflow_entries(int dtype, int stable, int first_log2w, int* idx) {
    int n = 0;
    for (int w = first_log2w; n < kMaxOverflow; ++w, ++n) {
        int found = -1;
        const auto& reg = registry();
        for (size_t i = 0; i < reg.size(); ++i)
            if (reg[i].dtype == dtype && reg[i].stable == stable && reg[i].lc >= 0 && reg[i].log2w == w &&
                (found < 0 || reg[i].lc < reg[size_t(found)].lc))
                found = int(i);
        if (found < 0) break;
        if (idx) idx[n] = found;
    }
    return n;
}

}  // namespace b200s

extern "C" {

int32_t b200s_ragged_max_length(b200s_dtype dtype, uint32_t flags) {
    if (dtype < 0 || dtype > 3) return 0;
    const int stable = effective_stable(dtype, flags);
    for (const RaggedEntry& e : ragged_registry())
        if (e.dtype == dtype && e.stable == stable) {
            const int top = kRaggedLmin + e.nb - 1;
            return int32_t(1) << (top + overflow_entries(dtype, stable, top + 1, nullptr));
        }
    return 0;
}

b200s_status b200s_plan_create(b200s_plan** out, b200s_dtype dtype, uint32_t flags, int64_t max_arrays,
                               int32_t device) {
    if (!out) return set_error(B200S_ERR_INVALID_ARGUMENT, "null plan pointer");
    *out = nullptr;
    if (dtype < 0 || dtype > 3) return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (max_arrays < 0 || max_arrays > 0x7ffffffeLL)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "max_arrays out of range");
    if (flags & ~(B200S_STABLE | B200S_SORTED_CHECK | B200S_PLAN_NO_GRAPH))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown flag bits");
    const int stable = effective_stable(dtype, flags);
    const RaggedEntry* rk = find_ragged(dtype, stable);
    if (!rk) return set_error(B200S_ERR_UNSUPPORTED, "no ragged kernel for this dtype");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return cuda_error(e, "multiprocessor count");
    const int per_sm = rk->resident_per_sm();
    if (per_sm <= 0) return set_error(B200S_ERR_CUDA, "ragged kernel does not fit on this device");
    auto* p = new b200s_plan();
    p->device = device;
    p->dtype = dtype;
    p->stable = stable;
    p->flags = flags;
    p->max_arrays = max_arrays;
    p->rk = rk;
    // The tile table (its packed rows and the ragged rows that set the masks
    // below) loads on the first lookup: make sure it has.
    int unused_form = 0;
    (void)lookup_default_entry(dtype, stable, 1, &unused_form);
    p->family_mask = ragged_family_mask(dtype, stable);
    p->dedicated_mask = ragged_dedicated_mask(dtype, stable);
    dedicated_entries(dtype, stable, rk->nb, &p->dedicated_mask, p->dedicated_entry, p->dedicated_xc);
    p->grid = sms * per_sm;
    p->bin_grid = sms * 4;
    const long long stride = std::max<long long>(1, max_arrays);
    p->spec.nb = rk->nb;
    p->spec.over_lo = kRaggedLmin + rk->nb;
    p->spec.n_over = overflow_entries(dtype, stable, p->spec.over_lo, p->over_entry);
    for (int i = 0; i < p->spec.n_over; ++i) p->over_xc[i] = cluster_xc(dtype, stable, p->over_entry[i]);
    p->spec.stride = int(stride);
    // control block, bucketed ids, plain ids, cluster-bucket ids
    const size_t ids_bytes = size_t(stride) * sizeof(int);
    e = cudaMalloc(&p->scratch, sizeof(RaggedCtl) + (2 + size_t(p->spec.n_over)) * ids_bytes);
    if (e != cudaSuccess) {
        delete p;
        return cuda_error(e, "plan scratch allocation");
    }
    p->ctl = static_cast<RaggedCtl*>(p->scratch);
    p->ids = reinterpret_cast<int*>(static_cast<char*>(p->scratch) + sizeof(RaggedCtl));
    p->plain_ids = p->ids + stride;
    p->oids = p->plain_ids + stride;
    e = cudaStreamCreateWithFlags(&p->capture, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
    for (int s = 0; s < b200s_plan::kSides && e == cudaSuccess; ++s) {
        e = cudaStreamCreateWithFlags(&p->side[s], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->join[s], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        b200s_plan_destroy(p);
        return cuda_error(e, "plan streams");
    }
    *out = p;
    return B200S_OK;
}

b200s_status b200s_plan_destroy(b200s_plan* p) {
    if (!p) return B200S_OK;
    cudaSetDevice(p->device);
    if (p->capture) cudaStreamSynchronize(p->capture);
    cudaDeviceSynchronize();
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->capture) cudaStreamDestroy(p->capture);
    for (int s = 0; s < b200s_plan::kSides; ++s) {
        if (p->side[s]) cudaStreamDestroy(p->side[s]);
        if (p->join[s]) cudaEventDestroy(p->join[s]);
    }
    if (p->fork) cudaEventDestroy(p->fork);
    if (p->scratch) cudaFree(p->scratch);
    delete p;
    return B200S_OK;
}

b200s_status b200s_sort_ragged(b200s_plan* p, const void* d_in, void* d_out, const int32_t* d_offsets,
                               int64_t arrays, void* stream) {
    if (!p) return set_error(B200S_ERR_INVALID_ARGUMENT, "null plan");
    if (arrays < 0 || arrays > p->max_arrays)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "arrays exceeds the plan's max_arrays");
    if (arrays == 0) return B200S_OK;
    if (!d_in || !d_out || !d_offsets) return set_error(B200S_ERR_INVALID_ARGUMENT, "null buffer");
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (p->flags & B200S_PLAN_NO_GRAPH) return record_sequence(p, d_in, d_out, d_offsets, int(arrays), st);
    if (!p->exec || p->g_in != d_in || p->g_out != d_out || p->g_off != d_offsets || p->g_arrays != arrays) {
        if (p->exec) {
            // the previous graph may still run on another stream
            cudaDeviceSynchronize();
            cudaGraphExecDestroy(p->exec);
            p->exec = nullptr;
        }
        e = cudaStreamBeginCapture(p->capture, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_error(e, "begin capture");
        b200s_status st_rec = record_sequence(p, d_in, d_out, d_offsets, int(arrays), p->capture);
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(p->capture, &graph);
        if (st_rec != B200S_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st_rec;
        }
        if (e != cudaSuccess) return cuda_error(e, "end capture");
        e = cudaGraphInstantiate(&p->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            p->exec = nullptr;
            return cuda_error(e, "graph instantiate");
        }
        p->g_in = d_in;
        p->g_out = d_out;
        p->g_off = d_offsets;
        p->g_arrays = arrays;
    }
    e = cudaGraphLaunch(p->exec, st);
    if (e != cudaSuccess) return cuda_error(e, "graph launch");
    return B200S_OK;
}

b200s_status b200s_sort_ragged_hinted(b200s_plan* p, const void* d_in, void* d_out, const int32_t* d_offsets,
                                      const int32_t* h_offsets, int64_t arrays, void* stream) {
    if (!p) return set_error(B200S_ERR_INVALID_ARGUMENT, "null plan");
    if (!h_offsets || !(p->flags & B200S_PLAN_NO_GRAPH))
        return b200s_sort_ragged(p, d_in, d_out, d_offsets, arrays, stream);
    if (arrays < 0 || arrays > p->max_arrays)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "arrays exceeds the plan's max_arrays");
    if (arrays == 0) return B200S_OK;
    if (!d_in || !d_out || !d_offsets) return set_error(B200S_ERR_INVALID_ARGUMENT, "null buffer");
    // the classes the batch holds, by the binning kernel's rule
    uint32_t present = 0, over_present = 0;
    for (int64_t a = 0; a < arrays; ++a) {
        const int n = h_offsets[a + 1] - h_offsets[a];
        if (n <= 0) continue;
        const int l = n <= 1 ? 0 : 32 - __builtin_clz(unsigned(n - 1));
        const int b = (l > kRaggedLmin ? l : kRaggedLmin) - kRaggedLmin;
        if (b < p->spec.nb) present |= 1u << b;
        else if (l - p->spec.over_lo < p->spec.n_over) over_present |= 1u << (l - p->spec.over_lo);
    }
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    return record_sequence(p, d_in, d_out, d_offsets, int(arrays), static_cast<cudaStream_t>(stream), present,
                           over_present);
}

b200s_status b200s_plan_too_long(b200s_plan* p, void* stream, int64_t* count) {
    if (!p || !count) return set_error(B200S_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    int v = 0;
    e = cudaMemcpyAsync(&v, &p->ctl->too_long, sizeof(int), cudaMemcpyDeviceToHost,
                        static_cast<cudaStream_t>(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_error(e, "read ragged status");
    *count = v;
    return B200S_OK;
}

}  // extern "C"

namespace {

// Groups the arrays on the host, uploads the id lists and records one launch
// per group: by exact length (by_bucket false: every array of a group has the
// same length) or by power-of-two working length (by_bucket true: the tile of
// W = 2^L sorts every array of length (W/2, W]; each array's own length comes
// from the offsets).
b200s_status prepare_plain(b200s_plan* p, const int32_t* h_offsets, int64_t arrays, bool by_bucket) {
    if (!p || (!h_offsets && arrays > 0)) return set_error(B200S_ERR_INVALID_ARGUMENT, "null argument");
    if (arrays < 0 || arrays > p->max_arrays)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "arrays exceeds the plan's max_arrays");
    auto key_of = [by_bucket](int n) { return by_bucket ? ceil_log2(n) : n; };
    // Counting sort of array ids by group key (empty arrays are skipped).
    int top = 0;
    for (int64_t a = 0; a < arrays; ++a) {
        const int n = h_offsets[a + 1] - h_offsets[a];
        if (n < 0) return set_error(B200S_ERR_INVALID_ARGUMENT, "offsets decrease");
        if (n > 0) top = std::max(top, key_of(n));
    }
    std::vector<int> start(size_t(top) + 2, 0);
    for (int64_t a = 0; a < arrays; ++a) {
        const int n = h_offsets[a + 1] - h_offsets[a];
        if (n > 0) ++start[size_t(key_of(n)) + 1];
    }
    for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
    std::vector<int> ids(size_t(std::max<int64_t>(arrays, 1)));
    std::vector<int> cursor(start.begin(), start.end() - 1);
    for (int64_t a = 0; a < arrays; ++a) {
        const int n = h_offsets[a + 1] - h_offsets[a];
        if (n > 0) ids[size_t(cursor[size_t(key_of(n))]++)] = int(a);
    }
    p->groups.clear();
    for (int k = by_bucket ? 0 : 1; k <= top; ++k) {
        const int c = start[size_t(k) + 1] - start[size_t(k)];
        if (!c) continue;
        const long long len = by_bucket ? (1LL << k) : k;
        int persistent = 0;
        const int entry = lookup_default_entry(p->dtype, p->stable, len, &persistent);
        if (entry < 0) return set_error(B200S_ERR_UNSUPPORTED, "array longer than the largest tile");
        p->groups.push_back({int(len), start[size_t(k)], c, entry, persistent});
    }
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess && arrays > 0)
        e = cudaMemcpy(p->plain_ids, ids.data(), size_t(arrays) * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "upload plain ids");
    return B200S_OK;
}

}  // namespace

extern "C" {

b200s_status b200s_plan_prepare_plain(b200s_plan* p, const int32_t* h_offsets, int64_t arrays) {
    return prepare_plain(p, h_offsets, arrays, false);
}

b200s_status b200s_plan_prepare_plain_buckets(b200s_plan* p, const int32_t* h_offsets, int64_t arrays) {
    return prepare_plain(p, h_offsets, arrays, true);
}

b200s_status b200s_sort_ragged_plain(b200s_plan* p, const void* d_in, void* d_out, const int32_t* d_offsets,
                                     void* stream) {
    if (!p || !d_in || !d_out || !d_offsets) return set_error(B200S_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (const auto& g : p->groups) {
        const KernelEntry& k = registry()[size_t(g.entry)];
        e = (g.persistent == 3 && k.launch_list_xc ? k.launch_list_xc : k.launch_list)(
            d_in, d_out, d_offsets, p->plain_ids + g.first, g.count, st);
        if (e != cudaSuccess) return cuda_error(e, "per-length launch");
    }
    return B200S_OK;
}

int32_t b200s_plan_plain_launches(const b200s_plan* p) { return p ? int32_t(p->groups.size()) : 0; }

}  // extern "C"
