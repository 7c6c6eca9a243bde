// C ABI of the batched sort: argument checking, tile selection, launches,
// and the host-buffer (end-to-end) entry point.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "b200sort.h"
#include "registry.h"
#include "xpose_registry.h"

namespace b200s {

namespace {
thread_local std::string g_error;
}

b200s_status set_error(b200s_status s, const std::string& msg) {
    g_error = msg;
    return s;
}

b200s_status cuda_error(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return set_error(e == cudaErrorMemoryAllocation ? B200S_ERR_OUT_OF_MEMORY : B200S_ERR_CUDA, m);
}

void clear_error() { g_error.clear(); }

size_t elem_bytes(int dtype) {
    switch (dtype) {
        case B200S_I32: return 4;
        case B200S_I32_I32: return 8;
        case B200S_U64: return 8;
        case B200S_U64_I32: return 16;
        default: return 0;
    }
}

// Keys alone are indistinguishable when equal: stable and unstable coincide.
int effective_stable(int dtype, uint32_t flags) {
    return ((flags & B200S_STABLE) && (dtype == B200S_I32_I32 || dtype == B200S_U64_I32)) ? 1 : 0;
}

int ceil_log2(long long n) {
    int b = 0;
    while ((1LL << b) < n) ++b;
    return b;
}

const std::vector<KernelEntry>& registry() {
    static std::vector<KernelEntry> all = [] {
        std::vector<KernelEntry> v;
        register_i32(v);
        register_rec(v);
        register_u64(v);
        register_cluster_keys(v);
        register_cluster_rec(v);
        register_cluster_u64rec(v);
        register_xc_keys(v);
        register_xc_rec(v);
        register_xc_cluster_rec(v);
        register_xc_u64rec(v);
        // single-warp tiles: launch form 3 over id lists is the one-warp
        // transposed network (xpose.cuh)
        for (KernelEntry& k : v)
            if (k.lw == 0 && k.lc < 0)
                for (const XposeEntry& x : xpose_registry())
                    if (x.dtype == k.dtype && x.stable == k.stable && x.lk == k.lk && x.lg == k.lg) {
                        k.launch_list_xc = x.launch_list;
                        k.launch_list_dev_xc = x.launch_list_dev;
                    }
        return v;
    }();
    return all;
}

namespace {

constexpr int kMaxLog2W = 20;

struct DefaultTable {
    int pick[4][2][kMaxLog2W + 1];        // registry index, -1 if none
    int persistent[4][2][kMaxLog2W + 1];  // launch form for that row
};

std::mutex g_table_mutex;

int preferred_lk(int dtype) { return dtype == B200S_I32 ? 5 : 4; }

DefaultTable build_defaults() {
    DefaultTable t;
    const auto& reg = registry();
    for (int d = 0; d < 4; ++d)
        for (int s = 0; s < 2; ++s)
            for (int w = 0; w <= kMaxLog2W; ++w) {
                int best = -1, best_score = -1;
                for (size_t i = 0; i < reg.size(); ++i) {
                    const KernelEntry& e = reg[i];
                    if (e.dtype != d || e.stable != s || e.log2w != w) continue;
                    // Prefer the type's preferred register depth, then fewer
                    // warps per array (fewer barriers); among cluster tiles,
                    // fewer CTAs per array (fewer distributed-shared-memory
                    // exchanges: the throughput choice).
                    int score = (e.lk == preferred_lk(d) ? 1000 : 100 * e.lk) - 10 * e.lw;
                    if (e.lc >= 0) score = 10000 - 100 * e.lc;
                    if (score > best_score) {
                        best_score = score;
                        best = int(i);
                    }
                }
                t.pick[d][s][w] = best;
                t.persistent[d][s][w] = 0;
            }
    return t;
}

struct TableRows {
    std::vector<std::array<int, 4>> packed;  // dtype*2+stable, log2w, registry index, persistent
    std::vector<std::array<int, 6>> ragged;  // dtype, stable, log2w, family, own tile (registry index or -1), form
};
b200s_status parse_table_file(const char* path, TableRows* out);
void apply_packed_rows(const TableRows& rows, DefaultTable& t);
std::string shipped_table_path();

}  // namespace

void set_ragged_family(int dtype, int stable, int log2w, int family, int own_entry, int own_form);

namespace {

DefaultTable& table() {
    static DefaultTable t = [] {
        DefaultTable d = build_defaults();
        const std::string path = shipped_table_path();
        TableRows rows;
        if (!path.empty() && std::ifstream(path).good() && parse_table_file(path.c_str(), &rows) == B200S_OK) {
            apply_packed_rows(rows, d);
            for (const auto& r : rows.ragged) set_ragged_family(r[0], r[1], r[2], r[3], r[4], r[5]);
        }
        clear_error();
        return d;
    }();
    return t;
}

// Entry for arrays of length n: the tabled tile for the smallest compiled
// working length >= n.
int lookup_default(int dtype, int stable, long long n, int* persistent) {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    const DefaultTable& t = table();
    for (int w = std::max(0, ceil_log2(n)); w <= kMaxLog2W; ++w)
        if (t.pick[dtype][stable][w] >= 0) {
            *persistent = t.persistent[dtype][stable][w];
            return t.pick[dtype][stable][w];
        }
    return -1;
}

int lookup_tile(int dtype, int stable, const b200s_tile& tile) {
    const auto& reg = registry();
    for (size_t i = 0; i < reg.size(); ++i) {
        const KernelEntry& e = reg[i];
        if (e.dtype == dtype && e.stable == stable && e.lk == tile.log2_items &&
            e.lg == tile.log2_lanes && e.lw == tile.log2_warps && std::max(e.lc, 0) == tile.log2_ctas)
            return int(i);
    }
    return -1;
}

void fill_tile(const KernelEntry& e, int persistent, b200s_tile* out) {
    out->log2_items = e.lk;
    out->log2_lanes = e.lg;
    out->log2_warps = e.lw;
    out->cta_threads = e.cta;
    out->persistent = persistent;
    out->log2_ctas = std::max(e.lc, 0);
}

bool valid_dtype(int d) { return d >= 0 && d <= 3; }

}  // namespace

namespace {

// Tile table CSV: '#' comments; packed rows dtype,flags,log2_w,log2_items,
// log2_lanes,log2_warps[,persistent[,log2_ctas]]; ragged rows
// r,dtype,flags,log2_w,family.
b200s_status parse_table_file(const char* path, TableRows* out) {
    std::ifstream f(path);
    if (!f) return set_error(B200S_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    std::string line;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
        std::replace(line.begin(), line.end(), ',', ' ');
        std::istringstream ss(line);
        const size_t first = line.find_first_not_of(" \t");
        if (line[first] == 'r') {
            std::string tag;
            int d, fl, w, fam;
            if (!(ss >> tag >> d >> fl >> w >> fam) || !valid_dtype(d) || w < 3 || w > 18 || fam < 0 || fam > 2)
                return set_error(B200S_ERR_INVALID_ARGUMENT,
                                 "tile table line " + std::to_string(lineno) + ": bad ragged row");
            const int stable = effective_stable(d, uint32_t(fl));
            // optional tile of the class's own launch (family 2): log2_items,
            // log2_lanes, log2_warps, form (0 or 3); a single-CTA tile of W
            int own = -1, form = 0, lk, lg, lw;
            if (ss >> lk) {
                if (!(ss >> lg >> lw >> form) || fam != 2 || (form != 0 && form != 3))
                    return set_error(B200S_ERR_INVALID_ARGUMENT,
                                     "tile table line " + std::to_string(lineno) + ": bad own-launch tile");
                own = lookup_tile(d, stable, b200s_tile{lk, lg, lw, 0, 0, 0});
                if (own < 0 || registry()[size_t(own)].log2w != w || registry()[size_t(own)].lc > 0)
                    return set_error(B200S_ERR_UNSUPPORTED,
                                     "tile table line " + std::to_string(lineno) + ": own-launch tile not compiled");
            }
            out->ragged.push_back({d, stable, w, fam, own, form});
            continue;
        }
        int d, fl, w, lk, lg, lw, pers = 0, lc = 0;
        if (!(ss >> d >> fl >> w >> lk >> lg >> lw))
            return set_error(B200S_ERR_INVALID_ARGUMENT,
                             "tile table line " + std::to_string(lineno) + ": expected 6 to 8 integers");
        if (!(ss >> pers)) pers = 0;
        else if (!(ss >> lc)) lc = 0;
        if (!valid_dtype(d) || w < 0 || w > kMaxLog2W)
            return set_error(B200S_ERR_INVALID_ARGUMENT,
                             "tile table line " + std::to_string(lineno) + ": bad dtype or log2_w");
        const int stable = effective_stable(d, uint32_t(fl));
        const b200s_tile tile{lk, lg, lw, 0, 0, lc};
        const int idx = lookup_tile(d, stable, tile);
        if (idx < 0 || registry()[size_t(idx)].log2w < w)
            return set_error(B200S_ERR_UNSUPPORTED,
                             "tile table line " + std::to_string(lineno) + ": tile not compiled or too short");
        if (pers < 0 || pers > 3)
            return set_error(B200S_ERR_INVALID_ARGUMENT,
                             "tile table line " + std::to_string(lineno) + ": launch form must be 0 .. 3");
        out->packed.push_back({d * 2 + stable, w, idx, pers});
    }
    return B200S_OK;
}

void apply_packed_rows(const TableRows& rows, DefaultTable& t) {
    for (const auto& u : rows.packed) {
        t.pick[u[0] / 2][u[0] % 2][u[1]] = u[2];
        t.persistent[u[0] / 2][u[0] % 2][u[1]] = u[3];
    }
}

// The tuned table shipped beside the library (tune/b200_table.csv next to
// libb200sort.so), or the file named by B200SORT_TILE_TABLE.
std::string shipped_table_path() {
    if (const char* env = std::getenv("B200SORT_TILE_TABLE")) return env;
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&b200s_version), &info) && info.dli_fname) {
        std::string lib = info.dli_fname;
        const size_t slash = lib.rfind('/');
        return (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/tune/b200_table.csv";
    }
    return std::string();
}

}  // namespace

int lookup_default_entry(int dtype, int stable, long long n, int* persistent) {
    return lookup_default(dtype, stable, n, persistent);
}

void set_ragged_family(int dtype, int stable, int log2w, int family, int own_entry, int own_form);

// The TMA-pipelined kernel for registry entry e and this batch, or null when
// the batch does not meet its requirements: whole 128-byte rows per array (at
// most 256), 16-byte aligned buffers, int32-addressable array indices.
const TmaEntry* tma_for(const KernelEntry& e, const void* in, const void* out, int n, long long arrays) {
    if (e.lw != 0 || e.lc >= 0) return nullptr;
    const long long bytes = (long long)n * (long long)elem_bytes(e.dtype);
    if (bytes % 128 != 0 || bytes / 128 > 256 || arrays > 0x7fffffffLL) return nullptr;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) return nullptr;
    for (const TmaEntry& t : tma_registry())
        if (t.dtype == e.dtype && t.stable == e.stable && t.lk == e.lk && t.lg == e.lg) return &t;
    return nullptr;
}

// The transposed-network kernel (launch form 3) for registry entry e, or null
// when none is compiled for its shape.
const XposeEntry* xpose_for(const KernelEntry& e) {
    if (e.lw != 0 || e.lc >= 0) return nullptr;
    for (const XposeEntry& x : xpose_registry())
        if (x.dtype == e.dtype && x.stable == e.stable && x.lk == e.lk && x.lg == e.lg) return &x;
    return nullptr;
}

// Launch the packed kernel of registry entry `idx`: form 0 one-shot, 1
// persistent with register prefetch, 2 persistent TMA pipeline, 3 transposed
// network (form 0 when the batch or the tile does not qualify).  opts:
// kOptSortedCheck (the sortedness test of B200S_SORTED_CHECK) is run by forms
// 0, 1 and 3; a form-2 request with it runs form 0, and the cluster kernels
// ignore it.
b200s_status launch_packed(int idx, int persistent, const void* in, void* out, int n,
                           long long arrays, cudaStream_t st, unsigned opts = 0) {
    const KernelEntry& e = registry()[size_t(idx)];
    if (persistent == 2 && (opts & kOptSortedCheck)) persistent = 0;
    if (persistent == 3) {
        const XposeEntry* x = xpose_for(e);
        if (x && ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) % uintptr_t(x->align)) != 0)
            x = nullptr;  // element-wide accesses need element-aligned buffers: form 0 instead
        if (x) {
            const cudaError_t err = x->launch(in, out, n, arrays, st, opts);
            if (err != cudaSuccess) return cuda_error(err, "transposed-network sort kernel launch");
            return B200S_OK;
        }
        if (!xpose_for(e) && e.launch_xc) {  // multi-warp and cluster tiles
            const cudaError_t err = e.launch_xc(in, out, n, arrays, 0, st, opts);
            if (err != cudaSuccess) return cuda_error(err, "transposed-network sort kernel launch");
            return B200S_OK;
        }
        persistent = 0;
    }
    if (persistent == 2) {
        if (const TmaEntry* t = tma_for(e, in, out, n, arrays)) {
            const cudaError_t err = t->launch(in, out, n, arrays, st);
            if (err != cudaSuccess) return cuda_error(err, "TMA sort kernel launch");
            return B200S_OK;
        }
        persistent = 0;
    }
    long long grid = (arrays + e.apc - 1) / e.apc;
    grid = std::min<long long>(grid, 0x7fffffffLL);
    cudaError_t err = persistent ? e.launch_pf(in, out, n, arrays, grid, st, opts)
                                 : e.launch(in, out, n, arrays, grid, st, opts);
    if (err != cudaSuccess) return cuda_error(err, "sort kernel launch");
    return B200S_OK;
}

// SMs of the current device (cached per device).
int sm_count() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    int v = cache[dev & 63].load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev & 63].store(v, std::memory_order_relaxed);
    }
    return v;
}

// The latency choice for a few long arrays: a cluster tile of the same
// working length with more, smaller CTAs per array, when every array's
// cluster is resident at once.  Clusters place within GPCs, so larger
// clusters leave SMs idle: on a 148-SM B200 (one 512-thread CTA per SM) 74
// 2-CTA, 33 4-CTA and 15 8-CTA clusters are resident, i.e. 100 %, 89 % and
// 81 % of the SMs; the rule allows arrays * CTAs per array up to that share.  The default cluster tile has the
// fewest CTAs per array (fewer distributed-shared-memory exchanges, the higher
// throughput once the batch fills the GPU); for one 65536-record array the
// 8-CTA tile halves the work per SM (87 us against 150 us on a B200).
int narrow_alternative(int idx, long long arrays) {
    const auto& reg = registry();
    const KernelEntry& e = reg[size_t(idx)];
    if (e.lc < 0 || arrays <= 0) return idx;
    int best = idx;
    for (size_t i = 0; i < reg.size(); ++i) {
        const KernelEntry& c = reg[i];
        if (c.dtype == e.dtype && c.stable == e.stable && c.log2w == e.log2w && c.lc > reg[size_t(best)].lc &&
            arrays * (1LL << c.lc) * 100 <= (c.lc <= 1 ? 100LL : c.lc == 2 ? 89LL : 81LL) * sm_count())
            best = int(i);
    }
    return best;
}

int select_entry(int dtype, uint32_t flags, long long n, const b200s_tile* tile, b200s_status* st,
                 int* persistent, long long arrays = -1) {
    const int stable = effective_stable(dtype, flags);
    int idx;
    *persistent = 0;
    if (tile) {
        *persistent = tile->persistent < 0 ? 0 : (tile->persistent > 3 ? 3 : tile->persistent);
        idx = lookup_tile(dtype, stable, *tile);
        if (idx < 0) {
            *st = set_error(B200S_ERR_UNSUPPORTED, "no compiled kernel for the requested tile");
            return -1;
        }
        if ((1LL << registry()[size_t(idx)].log2w) < n) {
            *st = set_error(B200S_ERR_UNSUPPORTED, "tile working length is shorter than n");
            return -1;
        }
    } else {
        idx = lookup_default(dtype, stable, n, persistent);
        if (idx < 0) {
            *st = set_error(B200S_ERR_UNSUPPORTED, "array length exceeds the largest compiled tile");
            return -1;
        }
        idx = narrow_alternative(idx, arrays);
    }
    *st = B200S_OK;
    return idx;
}

}  // namespace b200s

using namespace b200s;

extern "C" {

const char* b200s_version(void) { return "b200sort 0.1.0 (sm_100a)"; }

const char* b200s_status_string(b200s_status s) {
    switch (s) {
        case B200S_OK: return "ok";
        case B200S_ERR_INVALID_ARGUMENT: return "invalid argument";
        case B200S_ERR_UNSUPPORTED: return "unsupported";
        case B200S_ERR_CUDA: return "CUDA error";
        case B200S_ERR_OUT_OF_MEMORY: return "out of memory";
        case B200S_ERR_TIMEOUT: return "timeout";
        case B200S_ERR_BUDGET: return "over budget";
        case B200S_ERR_BUSY: return "busy";
        case B200S_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char* b200s_last_error(void) { return b200s::g_error.c_str(); }

int32_t b200s_max_length(b200s_dtype dtype, uint32_t flags) {
    if (!valid_dtype(dtype)) return 0;
    const int stable = effective_stable(dtype, flags);
    int best = 0;
    for (const KernelEntry& e : registry())
        if (e.dtype == dtype && e.stable == stable) best = std::max(best, e.log2w);
    return best ? int32_t(1) << best : 0;
}

int32_t b200s_tile_count(b200s_dtype dtype, uint32_t flags) {
    if (!valid_dtype(dtype)) return 0;
    const int stable = effective_stable(dtype, flags);
    int c = 0;
    for (const KernelEntry& e : registry())
        if (e.dtype == dtype && e.stable == stable) ++c;
    return c;
}

b200s_status b200s_tile_get(b200s_dtype dtype, uint32_t flags, int32_t index, b200s_tile* out) {
    if (!valid_dtype(dtype) || !out || index < 0)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "b200s_tile_get: bad argument");
    const int stable = effective_stable(dtype, flags);
    int c = 0;
    for (const KernelEntry& e : registry()) {
        if (e.dtype != dtype || e.stable != stable) continue;
        if (c++ == index) {
            fill_tile(e, 0, out);
            return B200S_OK;
        }
    }
    return set_error(B200S_ERR_INVALID_ARGUMENT, "b200s_tile_get: index out of range");
}

b200s_status b200s_default_tile(b200s_dtype dtype, uint32_t flags, int32_t n, b200s_tile* out) {
    if (!valid_dtype(dtype) || !out || n < 0)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "b200s_default_tile: bad argument");
    b200s_status st;
    int persistent = 0;
    const int idx = select_entry(dtype, flags, std::max(1, n), nullptr, &st, &persistent);
    if (idx < 0) return st;
    fill_tile(registry()[size_t(idx)], persistent, out);
    return B200S_OK;
}

b200s_status b200s_tile_info_get(b200s_dtype dtype, uint32_t flags, const b200s_tile* tile, int32_t n,
                                 b200s_tile_info* out) {
    if (!valid_dtype(dtype) || !out || n < 0)
        return set_error(B200S_ERR_INVALID_ARGUMENT, "b200s_tile_info_get: bad argument");
    b200s_status st;
    int persistent = 0;
    const int idx = select_entry(dtype, flags, std::max(1, n), tile, &st, &persistent);
    if (idx < 0) return st;
    const KernelEntry& e = registry()[size_t(idx)];
    cudaFuncAttributes a = {};
    const cudaError_t ce = e.attrs(&a);
    if (ce != cudaSuccess) return cuda_error(ce, "cudaFuncGetAttributes");
    int dev = 0, sm_threads = 2048, sm_regs = 65536, sm_smem = 228 * 1024, sm_blocks = 32;
    if (cudaGetDevice(&dev) == cudaSuccess) {
        cudaDeviceGetAttribute(&sm_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
        cudaDeviceGetAttribute(&sm_regs, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&sm_blocks, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    }
    // residency limits: threads, registers (allocated per warp in units of
    // 256), shared memory (plus 1 KB reserved per CTA), CTA slots
    const int warps = (e.cta + 31) / 32;
    const int regs_per_warp = ((a.numRegs * 32 + 255) / 256) * 256;
    const size_t smem = size_t(a.sharedSizeBytes) + e.smem + 1024;
    int active = std::min(sm_blocks, sm_threads / std::max(1, e.cta));
    if (regs_per_warp > 0) active = std::min(active, sm_regs / (regs_per_warp * warps));
    active = std::min<int>(active, int(size_t(sm_smem) / smem));
    out->registers_per_thread = a.numRegs;
    out->local_bytes_per_thread = int32_t(a.localSizeBytes);
    out->shared_bytes = int32_t(a.sharedSizeBytes + e.smem);
    out->cta_threads = e.cta;
    out->active_ctas_per_sm = active;
    out->working = int32_t(1) << e.log2w;
    out->arrays_per_cta = e.lc >= 0 ? 0 : e.apc;
    static const char aligned[16] = {};  // any 16-byte aligned address stands for the buffers
    out->tma_form = tma_for(e, aligned, aligned, std::max(1, n), 1) ? 1 : 0;
    out->xpose_form = (xpose_for(e) || e.launch_xc) ? 1 : 0;
    return B200S_OK;
}

b200s_status b200s_tma_timeouts(int64_t* count) {
    if (!count) return set_error(B200S_ERR_INVALID_ARGUMENT, "null count");
    const int64_t v = tma_timeouts();
    if (v < 0) return set_error(B200S_ERR_CUDA, "reading the TMA status word failed");
    *count = v;
    return B200S_OK;
}

b200s_status b200s_test_stall_tma_loads(int32_t enable) {
    if (!tma_set_extra_tx(enable ? 16u : 0u))
        return set_error(B200S_ERR_CUDA, "writing the TMA status word failed");
    return B200S_OK;
}

b200s_status b200s_load_tile_table(const char* path, int32_t* applied) {
    if (!path) return set_error(B200S_ERR_INVALID_ARGUMENT, "b200s_load_tile_table: null path");
    TableRows rows;
    b200s_status st = parse_table_file(path, &rows);
    if (st != B200S_OK) return st;
    table();  // the built-in defaults and the shipped table come first
    {
        std::lock_guard<std::mutex> lock(g_table_mutex);
        apply_packed_rows(rows, table());
    }
    for (const auto& r : rows.ragged) set_ragged_family(r[0], r[1], r[2], r[3], r[4], r[5]);
    if (applied) *applied = int32_t(rows.packed.size() + rows.ragged.size());
    clear_error();
    return B200S_OK;
}

b200s_status b200s_sort_packed(b200s_dtype dtype, const void* d_in, void* d_out, int32_t n,
                               int64_t arrays, uint32_t flags, const b200s_tile* tile,
                               void* stream) {
    if (!valid_dtype(dtype)) return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (n < 0 || arrays < 0) return set_error(B200S_ERR_INVALID_ARGUMENT, "negative n or arrays");
    if (flags & ~(B200S_STABLE | B200S_SORTED_CHECK))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown flag bits");
    if (n == 0 || arrays == 0) return B200S_OK;
    if (!d_in || !d_out) return set_error(B200S_ERR_INVALID_ARGUMENT, "null buffer");
    b200s_status st;
    int persistent = 0;
    const int idx = select_entry(dtype, flags, n, tile, &st, &persistent, arrays);
    if (idx < 0) return st;
    return launch_packed(idx, persistent, d_in, d_out, n, arrays, static_cast<cudaStream_t>(stream),
                         (flags & B200S_SORTED_CHECK) ? kOptSortedCheck : 0u);
}

}  // extern "C"

// ---- sessions: host buffers in, host buffers out -------------------------------
// One copy-in stream carries each chunk's host-to-device copy followed by its
// sort; one copy-out stream copies each sorted chunk back once the sort's
// event fires.  kSlots device buffers form a ring: chunk k uses slot k % kSlots
// and its copy-in waits for the copy-out of chunk k - kSlots.
struct b200s_session {
    int device = 0;
    static constexpr int kSlots = 4;
    cudaStream_t in = nullptr, out = nullptr;
    cudaEvent_t sorted[kSlots] = {}, freed[kSlots] = {};
    void* dbuf[kSlots] = {};
    size_t capacity = 0;  // bytes per slot
};

namespace {

void release_buffers(b200s_session* s) {
    for (int i = 0; i < b200s_session::kSlots; ++i) {
        if (s->dbuf[i]) cudaFree(s->dbuf[i]);
        s->dbuf[i] = nullptr;
    }
    s->capacity = 0;
}

void release_session(b200s_session* s) {
    if (s->in) cudaStreamSynchronize(s->in);
    if (s->out) cudaStreamSynchronize(s->out);
    release_buffers(s);
    for (int i = 0; i < b200s_session::kSlots; ++i) {
        if (s->sorted[i]) cudaEventDestroy(s->sorted[i]);
        if (s->freed[i]) cudaEventDestroy(s->freed[i]);
    }
    if (s->in) cudaStreamDestroy(s->in);
    if (s->out) cudaStreamDestroy(s->out);
    delete s;
}

}  // namespace

extern "C" {

b200s_status b200s_session_create(b200s_session** out, int32_t device) {
    if (!out) return set_error(B200S_ERR_INVALID_ARGUMENT, "null session pointer");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    auto* s = new b200s_session();
    s->device = device;
    e = cudaStreamCreateWithFlags(&s->in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->out, cudaStreamNonBlocking);
    for (int i = 0; i < b200s_session::kSlots && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&s->sorted[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->freed[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        release_session(s);
        return cuda_error(e, "session streams and events");
    }
    *out = s;
    return B200S_OK;
}

b200s_status b200s_session_destroy(b200s_session* s) {
    if (!s) return B200S_OK;
    cudaSetDevice(s->device);
    release_session(s);
    return B200S_OK;
}

b200s_status b200s_sort_packed_host(b200s_session* s, b200s_dtype dtype, const void* h_in,
                                    void* h_out, int32_t n, int64_t arrays, uint32_t flags) {
    if (!s) return set_error(B200S_ERR_INVALID_ARGUMENT, "null session");
    if (!valid_dtype(dtype)) return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (n < 0 || arrays < 0) return set_error(B200S_ERR_INVALID_ARGUMENT, "negative n or arrays");
    if (flags & ~(B200S_STABLE | B200S_SORTED_CHECK))
        return set_error(B200S_ERR_INVALID_ARGUMENT, "unknown flag bits");
    if (n == 0 || arrays == 0) return B200S_OK;
    if (!h_in || !h_out) return set_error(B200S_ERR_INVALID_ARGUMENT, "null buffer");
    b200s_status st;
    int persistent = 0;
    const int idx = select_entry(dtype, flags, n, nullptr, &st, &persistent);
    if (idx < 0) return st;
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");

    // A quarter of the batch per chunk, within 2..64 MB of whole arrays.
    // Four chunks overlap the copy-out of one with the copy-in of the next
    // while keeping each copy large: on a PCIe Gen5 B200 a 16.8 MB batch
    // took 495 us this way against 580 us with 2 MB chunks on three
    // in-order streams (interleaved small copies in both directions lose
    // about 15 us per pair).
    const size_t eb = elem_bytes(dtype);
    const size_t array_bytes = size_t(n) * eb;
    const size_t total = size_t(arrays) * array_bytes;
    const size_t target = std::min<size_t>(size_t(64) << 20, std::max<size_t>(size_t(2) << 20, total / 4));
    const long long per_chunk = std::max<long long>(1, (long long)(target / array_bytes));
    const size_t need = size_t(std::min<long long>(per_chunk, arrays)) * array_bytes;
    if (need > s->capacity) {
        cudaStreamSynchronize(s->in);
        cudaStreamSynchronize(s->out);
        release_buffers(s);
        for (int i = 0; i < b200s_session::kSlots; ++i) {
            e = cudaMalloc(&s->dbuf[i], need);
            if (e != cudaSuccess) {
                release_buffers(s);
                return cuda_error(e, "session buffer allocation");
            }
        }
        s->capacity = need;
    }
    const char* src = static_cast<const char*>(h_in);
    char* dst = static_cast<char*>(h_out);
    // On a failure part way, wait for the copies already queued so that none
    // touches the caller's buffers after the call returns.
    auto drain = [s](b200s_status status) {
        cudaStreamSynchronize(s->in);
        cudaStreamSynchronize(s->out);
        return status;
    };
    long long chunk = 0;
    for (long long first = 0; first < arrays; first += per_chunk, ++chunk) {
        const long long count = std::min<long long>(per_chunk, arrays - first);
        const size_t bytes = size_t(count) * array_bytes;
        const int k = int(chunk % b200s_session::kSlots);
        // the slot's previous chunk must have left before this one lands
        e = cudaStreamWaitEvent(s->in, s->freed[k], 0);
        if (e != cudaSuccess) return drain(cuda_error(e, "session slot wait"));
        e = cudaMemcpyAsync(s->dbuf[k], src + size_t(first) * array_bytes, bytes, cudaMemcpyHostToDevice, s->in);
        if (e != cudaSuccess) return drain(cuda_error(e, "host-to-device copy"));
        st = launch_packed(idx, persistent, s->dbuf[k], s->dbuf[k], n, count, s->in,
                           (flags & B200S_SORTED_CHECK) ? kOptSortedCheck : 0u);
        if (st != B200S_OK) return drain(st);
        e = cudaEventRecord(s->sorted[k], s->in);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s->out, s->sorted[k], 0);
        if (e != cudaSuccess) return drain(cuda_error(e, "session sort event"));
        e = cudaMemcpyAsync(dst + size_t(first) * array_bytes, s->dbuf[k], bytes, cudaMemcpyDeviceToHost, s->out);
        if (e != cudaSuccess) return drain(cuda_error(e, "device-to-host copy"));
        e = cudaEventRecord(s->freed[k], s->out);
        if (e != cudaSuccess) return drain(cuda_error(e, "session slot event"));
    }
    e = cudaStreamSynchronize(s->in);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->out);
    if (e != cudaSuccess) return cuda_error(e, "session synchronize");
    return B200S_OK;
}

}  // extern "C"
