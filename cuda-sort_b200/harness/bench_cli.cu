// b200sort_bench: the reference's `bench` command line and CSV schema
// (bench.cu:66-136, 230-271), driving b200sort and the baselines on one GPU.
//
// Options, their defaults and checks, the size sweep (bench.cu:587-598), the
// per-size array count (bench.cu:600-608), the nine input distributions with
// EXTREMES added under --check-only (bench.cu:159-192, 630), the record
// validation (bench.cu:204-228), the timing protocol (restore, then CUDA
// events around the launch plus the wall clock, bench.cu:320-352), the PASS
// lines and the CSV columns are the reference's, so that its result files and
// plotting scripts read these files unchanged.  Columns appended after the
// reference's: keys_per_s, hbm_bytes, roofline_frac, tile.
//
// Methods:
//   b200_bitonic         b200sort with its tabled tile for n (the product)
//   b200_tiles           every compiled tile that covers n, both launch forms
//   b200_ragged          the same batch as CSR arrays through a ragged plan
//   cub_block_merge      CUB BlockMergeSort, the reference's thread sweep
//   thrust_segment_loop  one thrust::sort per array
//   bitonic_warp, bitonic_v1 .. bitonic_v6_register
//                        the reference's method names, run as b200sort's
//                        tabled tile (its Sorted/Shared/Async switches do not
//                        change the output; their columns read -1)
//   large_partition, large_merge, large_hybrid (--mode large)
//                        one array per batch through b200sort (thread-block
//                        clusters), up to b200s_max_length
// An empty --methods runs the b200_*, cub and thrust methods.
#include <cuda_runtime.h>
#include <cub/version.cuh>
#include <thrust/version.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "b200sort.h"

extern "C" int cub_block_merge_sort(int dtype, void* d, int n, int arrays, int working, int threads, void* stream);
extern "C" int thrust_segment_sort(int dtype, void* d, int n, int arrays, void* stream);

namespace {

struct Rec {
    int key;
    int data;
};

template <class T> constexpr b200s_dtype dtype_of() { return std::is_same<T, Rec>::value ? B200S_I32_I32 : B200S_I32; }
template <class T> __host__ __device__ int key_of(const T& v) {
    if constexpr (std::is_same<T, Rec>::value) return v.key; else return v;
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void check_b200(b200s_status s, const char* what) {
    if (s != B200S_OK)
        throw std::runtime_error(std::string(what) + ": " + b200s_status_string(s) + ": " + b200s_last_error());
}

// ---- options (bench.cu:44-136) ----------------------------------------------------
struct Options {
    std::string mode = "small", type = "both", prefix;
    int minSize = 1, maxSize = 0, maxThreads = 1024, arrays = 4096, batchElements = 1 << 22, repetitions = 5;
    bool checkOnly = false;
    double hbmGBs = 6541.1;  // measured copy bandwidth of this pool's B200s
    std::set<std::string> methods;
    bool explicitly(const char* m) const { return methods.count(m) != 0; }
    bool enabled(const char* m) const { return methods.empty() || methods.count(m) != 0; }
};

const std::set<std::string> kLegacy = {"bitonic_warp",   "bitonic_v1",        "bitonic_v2",         "bitonic_v3",
                                       "bitonic_v4_xor", "bitonic_v5_static", "bitonic_v6_register"};
const std::set<std::string> kLarge = {"large_partition", "large_merge", "large_hybrid"};

std::string timestamp() {
    const auto now = std::time(nullptr);
    char v[32];
    std::strftime(v, sizeof(v), "%Y-%m-%d-%H-%M-%S", std::localtime(&now));
    return v;
}

void usage() {
    std::cout << "Usage: b200sort_bench [--mode small|large|both] [--type int|record|both]\n"
                 "  --min-size N       Minimum array length (default 1)\n"
                 "  --max-size N       Maximum array length (default: the reference's bitonic capacity,\n"
                 "                     4096 int / 2048 record; up to b200s_max_length)\n"
                 "  --max-threads T    CUB thread sweep bound, a multiple of 32 in [32,1024] (default 1024)\n"
                 "  --arrays A         Maximum independent arrays per small batch (default 4096)\n"
                 "  --batch-elements M Bound N*A per batch (default 4194304)\n"
                 "  --repetitions R    Timed repetitions after warm-up (default 5)\n"
                 "  --output PREFIX    CSV path prefix\n"
                 "  --methods LIST     Comma-separated method names (default: b200_bitonic, b200_tiles,\n"
                 "                     b200_ragged, cub_block_merge, thrust_segment_loop); the reference's\n"
                 "                     bitonic_* and large_* names run b200sort's tabled tile\n"
                 "  --hbm-gbs G        HBM bandwidth for roofline_frac (default 6541.1 GB/s)\n"
                 "  --check-only       Validate every configuration on 3 arrays, no timing, EXTREMES added\n"
                 "Small CSV: E_s is the CUDA-event batch time, X_s = E_s/(A*N*log2 N) (N=1: nan).\n";
}

Options parse(int argc, char** argv) {
    Options o;
    o.prefix = "benchmark_" + timestamp();
    for (int i = 1; i < argc; ++i) {
        const std::string key = argv[i];
        if (key == "--check-only") {
            o.checkOnly = true;
            continue;
        }
        if (i + 1 >= argc) throw std::runtime_error("Missing value for " + key);
        const std::string value = argv[++i];
        if (key == "--mode") o.mode = value;
        else if (key == "--type") o.type = value;
        else if (key == "--output") o.prefix = value;
        else if (key == "--hbm-gbs") o.hbmGBs = std::stod(value);
        else if (key == "--methods") {
            std::istringstream names(value);
            std::string m;
            while (std::getline(names, m, ',')) {
                if (m.empty()) throw std::runtime_error("Empty name in --methods");
                o.methods.insert(m);
            }
            if (o.methods.empty() || value.back() == ',') throw std::runtime_error("Empty name in --methods");
        } else {
            size_t used = 0;
            const long long v = std::stoll(value, &used);
            if (used != value.size() || v < 1 || v > (1 << 28))
                throw std::runtime_error("Invalid positive integer for " + key);
            const int n = int(v);
            if (key == "--min-size") o.minSize = n;
            else if (key == "--max-size") o.maxSize = n;
            else if (key == "--max-threads") o.maxThreads = n;
            else if (key == "--arrays") o.arrays = n;
            else if (key == "--batch-elements") o.batchElements = n;
            else if (key == "--repetitions") o.repetitions = n;
            else throw std::runtime_error("Unknown option: " + key);
        }
    }
    if (o.mode != "small" && o.mode != "large" && o.mode != "both") throw std::runtime_error("Invalid --mode");
    if (o.type != "int" && o.type != "record" && o.type != "both") throw std::runtime_error("Invalid --type");
    if (o.maxThreads < 32 || o.maxThreads > 1024 || o.maxThreads % 32)
        throw std::runtime_error("--max-threads must be a multiple of 32 in [32,1024]");
    if (o.maxSize && o.minSize > o.maxSize) throw std::runtime_error("--min-size exceeds --max-size");
    std::set<std::string> known = {"b200_bitonic", "b200_tiles", "b200_ragged", "cub_block_merge",
                                   "thrust_segment_loop"};
    known.insert(kLegacy.begin(), kLegacy.end());
    known.insert(kLarge.begin(), kLarge.end());
    for (const auto& m : o.methods)
        if (!known.count(m)) throw std::runtime_error("Unknown --methods entry: " + m);
    if (o.checkOnly) {
        o.arrays = std::min(o.arrays, 3);
        o.repetitions = 0;
    }
    return o;
}

// ---- inputs (bench.cu:24-41, 152-202) ----------------------------------------------
enum Dist { SORTED, REVERSED, RANDOM, NORMAL, CONSTANT, BINARY, PERTURBED_2, PERTURBED_8, PERTURBED_32, EXTREMES };
const char* kDistNames[] = {"SORTED",      "REVERSED",    "RANDOM",       "NORMAL",  "CONSTANT",
                            "BINARY",      "PERTURBED_2", "PERTURBED_8",  "PERTURBED_32", "EXTREMES"};
int amplitude(int d) { return d == PERTURBED_2 ? 2 : d == PERTURBED_8 ? 8 : d == PERTURBED_32 ? 32 : 0; }

// The reference's stateless integer hash, so that every method (and the
// reference's own bench) sees the same keys.
__host__ __device__ inline unsigned hash32(unsigned x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    return x ^ (x >> 16);
}

template <class T>
__global__ void k_generate(T* data, int n, int count, int dist) {
    for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < count; i += int(gridDim.x * blockDim.x)) {
        const int j = i % n;
        const unsigned r = hash32(unsigned(i) + 1234U);
        int key;
        if (dist == SORTED || dist == PERTURBED_2 || dist == PERTURBED_8 || dist == PERTURBED_32) key = j;
        else if (dist == REVERSED) key = n - 1 - j;
        else if (dist == RANDOM) key = int(r % 1000001U);
        else if (dist == NORMAL) {
            const float u = (float(r & 0xffffffU) + 1.0f) / 16777217.0f;
            const float v = float(hash32(r) & 0xffffffU) / 16777216.0f;
            const float z = sqrtf(-2.0f * logf(u)) * cosf(6.28318530718f * v);
            key = int(z * (1.0f + n / 4.0f) + n / 2.0f);
            key = key < 0 ? 0 : (key > n ? n : key);
        } else if (dist == CONSTANT) key = 99;
        else if (dist == BINARY) key = j % 2;
        else {
            const int ex[] = {INT_MAX, INT_MIN, 0, INT_MAX, -1, 1};
            key = ex[j % 6];
        }
        if constexpr (std::is_same<T, Rec>::value) data[i] = Rec{key, i};
        else data[i] = key;
    }
}

// Keys must equal the host-sorted reference; records must also carry their
// own payload (= input position), from their own array, each exactly once.
template <class T>
__global__ void k_validate(const T* input, const T* result, const T* expect, int n, int count, int* seen,
                           int* error) {
    for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < count; i += int(gridDim.x * blockDim.x)) {
        bool ok = key_of(result[i]) == key_of(expect[i]);
        if constexpr (std::is_same<T, Rec>::value) {
            const int o = result[i].data;
            if (o < 0 || o >= count || o / n != i / n) ok = false;
            else {
                if (input[o].key != result[i].key || input[o].data != result[i].data) ok = false;
                if (atomicAdd(seen + o, 1) != 0) ok = false;
            }
        }
        if (!ok) atomicExch(error, 1);
    }
}

template <class T> struct Dev {
    T* p = nullptr;
    explicit Dev(size_t count) { check_cuda(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc"); }
    ~Dev() { cudaFree(p); }
    Dev(const Dev&) = delete;
    Dev& operator=(const Dev&) = delete;
};

// ---- CSV (bench.cu:230-271, columns appended) ----------------------------------------
struct Config {
    std::string method;
    int testSorted = -1, fullSM = -1, asyncCopy = -1;
    int threads = 0, items = 0, working = 0;
    long long shared = 0;
    int regs = -1, active = -1;
    long long local = -1;
    std::string tile;
};

struct Csv {
    std::ofstream out;
    int runtime = 0;
    double hbm;
    Csv(const std::string& path, double hbm_gbs) : hbm(hbm_gbs) {
        const auto parent = std::filesystem::path(path).parent_path();
        if (!parent.empty()) std::filesystem::create_directories(parent);
        out.open(path);
        if (!out) throw std::runtime_error("Cannot open " + path);
        check_cuda(cudaRuntimeGetVersion(&runtime), "cudaRuntimeGetVersion");
        out << "method,distribution,N,arrays,total_values,working_values,threads,items_per_thread,"
               "testsorted,fullsm,asynccpy,shared_bytes,trial,E_s,X_s,E_wall_s,"
               "wall_X_s,time_per_array_s,time_per_value_s,validated,cuda_runtime,thrust_version,cub_version,"
               "registers_per_thread,active_blocks_per_sm,local_bytes_per_thread,"
               "keys_per_s,hbm_bytes,roofline_frac,tile\n";
        out << std::setprecision(17);
    }
    void write(const Config& c, int dist, int n, int arrays, int trial, double e, double wall, size_t elem) {
        const double values = double(n) * arrays;
        const double denom = n > 1 ? values * std::log2(double(n)) : 0;
        const double nan = std::numeric_limits<double>::quiet_NaN();
        const double bytes = 2.0 * values * double(elem);
        out << c.method << ',' << kDistNames[dist] << ',' << n << ',' << arrays << ',' << size_t(n) * arrays << ','
            << c.working << ',' << c.threads << ',' << c.items << ',' << c.testSorted << ',' << c.fullSM << ','
            << c.asyncCopy << ',' << c.shared << ',' << trial << ',' << e << ',' << (denom ? e / denom : nan)
            << ',' << wall << ',' << (denom ? wall / denom : nan) << ',' << e / arrays << ',' << e / values
            << ",1," << runtime << ',' << THRUST_VERSION << ',' << CUB_VERSION << ',' << c.regs << ','
            << c.active << ',' << c.local << ',' << values / e << ',' << bytes << ','
            << (bytes / (hbm * 1e9)) / e << ',' << c.tile << '\n';
        out.flush();
    }
};

// ---- one batch: inputs, host reference, timing, validation (bench.cu:273-352) --------
template <class T> struct Batch {
    int n, arrays, count, dist;
    const Options& opt;
    Csv& csv;
    Dev<T> input, values, expect;
    Dev<int> seen, error;
    cudaEvent_t e0, e1;

    Batch(int n_, int arrays_, int d, const Options& o, Csv& c)
        : n(n_), arrays(arrays_), count(n_ * arrays_), dist(d), opt(o), csv(c), input(size_t(count)),
          values(size_t(count)), expect(size_t(count)),
          seen(std::is_same<T, Rec>::value ? size_t(count) : 1), error(1) {
        check_cuda(cudaEventCreate(&e0), "event");
        check_cuda(cudaEventCreate(&e1), "event");
        k_generate<<<256, 256>>>(input.p, n, count, dist);
        check_cuda(cudaGetLastError(), "generate");
        std::vector<T> host(static_cast<size_t>(count));
        check_cuda(cudaMemcpy(host.data(), input.p, size_t(count) * sizeof(T), cudaMemcpyDeviceToHost), "D2H");
        if (const int amp = amplitude(dist)) {
            // x[i] = 4i + U{-4r..4r} per array, seeded by the array index
            // (bench_distributions.hpp:11-19, bench.cu:290-297)
            for (int a = 0; a < arrays; ++a) {
                std::mt19937 rng(hash32(unsigned(a) + 1234U));
                std::uniform_int_distribution<int> noise(-4 * amp, 4 * amp);
                for (int i = 0; i < n; ++i) {
                    const int key = 4 * i + noise(rng);
                    T& v = host[size_t(a) * n + i];
                    if constexpr (std::is_same<T, Rec>::value) v.key = key; else v = key;
                }
            }
            check_cuda(cudaMemcpy(input.p, host.data(), size_t(count) * sizeof(T), cudaMemcpyHostToDevice), "H2D");
        }
        for (int a = 0; a < arrays; ++a)
            std::sort(host.begin() + size_t(a) * n, host.begin() + size_t(a + 1) * n,
                      [](const T& x, const T& y) { return key_of(x) < key_of(y); });
        check_cuda(cudaMemcpy(expect.p, host.data(), size_t(count) * sizeof(T), cudaMemcpyHostToDevice), "H2D");
    }
    ~Batch() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    void restore() {
        check_cuda(cudaMemcpyAsync(values.p, input.p, size_t(count) * sizeof(T), cudaMemcpyDeviceToDevice), "restore");
        check_cuda(cudaDeviceSynchronize(), "restore sync");
    }
    void verify(const Config& c) {
        check_cuda(cudaMemset(seen.p, 0, sizeof(int) * (std::is_same<T, Rec>::value ? size_t(count) : 1)), "memset");
        check_cuda(cudaMemset(error.p, 0, sizeof(int)), "memset");
        k_validate<<<256, 256>>>(input.p, values.p, expect.p, n, count, seen.p, error.p);
        check_cuda(cudaGetLastError(), "validate");
        int failed = 0;
        check_cuda(cudaMemcpy(&failed, error.p, sizeof(int), cudaMemcpyDeviceToHost), "validate D2H");
        if (failed)
            throw std::runtime_error("Validation failed: " + c.method + " N=" + std::to_string(n) +
                                     " threads=" + std::to_string(c.threads) + " tile=" + c.tile +
                                     " distribution=" + kDistNames[dist]);
    }
    // launch() returns false when the configuration cannot run (skipped).
    void run(const Config& c, const std::function<bool()>& launch) {
        restore();
        if (!launch()) return;
        check_cuda(cudaGetLastError(), "launch");
        check_cuda(cudaDeviceSynchronize(), "sync");
        verify(c);
        if (opt.checkOnly) {
            std::cout << "PASS " << c.method << " N=" << n << " threads=" << c.threads << " sorted=" << c.testSorted
                      << " fullsm=" << c.fullSM << " async=" << c.asyncCopy << ' ' << kDistNames[dist]
                      << (c.tile.empty() ? "" : " tile=" + c.tile) << '\n';
            return;
        }
        for (int trial = 0; trial < opt.repetitions; ++trial) {
            restore();
            const auto t0 = std::chrono::steady_clock::now();
            check_cuda(cudaEventRecord(e0), "event");
            launch();
            check_cuda(cudaGetLastError(), "launch");
            check_cuda(cudaEventRecord(e1), "event");
            check_cuda(cudaEventSynchronize(e1), "event sync");
            const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            float ms = 0;
            check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
            verify(c);
            csv.write(c, dist, n, arrays, trial, double(ms) * 1e-3, wall, sizeof(T));
        }
    }
};

std::string tile_name(const b200s_tile& t) {
    std::ostringstream s;
    s << "K" << (1 << t.log2_items) << "/G" << (1 << t.log2_lanes) << "/W" << (1 << t.log2_warps) << "/C"
      << (1 << t.log2_ctas) << (t.persistent ? "/pf" : "");
    return s.str();
}

template <class T> Config b200_config(const std::string& method, int n, const b200s_tile* tile) {
    Config c;
    c.method = method;
    b200s_tile t;
    if (tile) t = *tile;
    else check_b200(b200s_default_tile(dtype_of<T>(), 0, n, &t), "b200s_default_tile");
    b200s_tile_info info;
    check_b200(b200s_tile_info_get(dtype_of<T>(), 0, tile, n, &info), "b200s_tile_info_get");
    c.threads = info.cta_threads;
    c.items = 1 << t.log2_items;
    c.working = info.working;
    c.shared = info.shared_bytes;
    c.regs = info.registers_per_thread;
    c.active = info.active_ctas_per_sm;
    c.local = info.local_bytes_per_thread;
    c.tile = tile_name(t);
    return c;
}

template <class T> bool sort_b200(Batch<T>& b, const b200s_tile* tile) {
    check_b200(b200s_sort_packed(dtype_of<T>(), b.values.p, b.values.p, b.n, b.arrays, 0, tile, nullptr),
               "b200s_sort_packed");
    return true;
}

int working_of(int n) {
    int w = 32;
    while (w < n) w *= 2;
    return w;
}

// The reference's bitonic capacity: 48 KB of shared memory for two buffers
// (cusort.hpp:231-237): 4096 int, 2048 records.
template <class T> int reference_capacity() { return std::is_same<T, Rec>::value ? 2048 : 4096; }

template <class T> void small_methods(Batch<T>& b, const Options& o) {
    const int n = b.n;
    if (o.enabled("b200_bitonic")) {
        const Config c = b200_config<T>("b200_bitonic", n, nullptr);
        b.run(c, [&] { return sort_b200(b, nullptr); });
    }
    for (const std::string& m : kLegacy) {
        if (!o.explicitly(m.c_str())) continue;
        if (m == "bitonic_warp" && n > 32) continue;
        if (m != "bitonic_warp" && n < 32) continue;
        const Config c = b200_config<T>(m, n, nullptr);
        b.run(c, [&] { return sort_b200(b, nullptr); });
    }
    if (o.enabled("b200_tiles")) {
        const int count = b200s_tile_count(dtype_of<T>(), 0);
        for (int i = 0; i < count; ++i) {
            b200s_tile t;
            check_b200(b200s_tile_get(dtype_of<T>(), 0, i, &t), "b200s_tile_get");
            const int w = 1 << (t.log2_items + t.log2_lanes + t.log2_warps + t.log2_ctas);
            if (w < n || w > 4 * std::max(8, working_of(n))) continue;
            for (int pf = 0; pf < 2; ++pf) {
                if (pf && t.log2_ctas) continue;
                t.persistent = pf;
                const Config c = b200_config<T>("b200_tiles", n, &t);
                b.run(c, [&] { return sort_b200(b, &t); });
            }
        }
    }
    if (o.enabled("b200_ragged") && n <= b200s_ragged_max_length(dtype_of<T>(), 0)) {
        std::vector<int> off(size_t(b.arrays) + 1);
        for (int a = 0; a <= b.arrays; ++a) off[size_t(a)] = a * n;
        Dev<int> d_off(off.size());
        check_cuda(cudaMemcpy(d_off.p, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice), "offsets");
        b200s_plan* plan = nullptr;
        check_b200(b200s_plan_create(&plan, dtype_of<T>(), 0, b.arrays, 0), "b200s_plan_create");
        Config c;
        c.method = "b200_ragged";
        c.working = working_of(n);
        c.tile = "bucketed";
        try {
            b.run(c, [&] {
                check_b200(b200s_sort_ragged(plan, b.values.p, b.values.p, d_off.p, b.arrays, nullptr),
                           "b200s_sort_ragged");
                return true;
            });
        } catch (...) {
            b200s_plan_destroy(plan);
            throw;
        }
        b200s_plan_destroy(plan);
    }
    if (o.enabled("cub_block_merge")) {
        const int w = working_of(n);
        const int cap = reference_capacity<T>();
        for (int threads = 32; threads <= std::min(w, o.maxThreads); threads *= 2) {
            const int items = w / threads;
            if (w > cap || items > 32 || items * threads != w) continue;  // compiled: items <= 32
            Config c;
            c.method = "cub_block_merge";
            c.threads = threads;
            c.items = items;
            c.working = w;
            b.run(c, [&] {
                return cub_block_merge_sort(std::is_same<T, Rec>::value ? 1 : 0, b.values.p, n, b.arrays, w,
                                            threads, nullptr) == 0;
            });
        }
    }
    if (o.enabled("thrust_segment_loop")) {
        Config c;
        c.method = "thrust_segment_loop";
        c.working = n;
        b.run(c, [&] {
            return thrust_segment_sort(std::is_same<T, Rec>::value ? 1 : 0, b.values.p, n, b.arrays, nullptr) == 0;
        });
    }
}

std::vector<int> small_sizes(int lo, int hi) {  // bench.cu:587-598
    std::set<int> s;
    for (int n = 1; n <= std::min(32, hi); ++n) s.insert(n);
    for (int n = 64; n <= std::min(1024, hi); n += 32) s.insert(n);
    for (int n = 32; n <= hi; n *= 2)
        for (int d : {-1, 0, 1})
            if (n + d >= 1 && n + d <= hi) s.insert(n + d);
    s.insert(hi);
    std::vector<int> out;
    for (int n : s)
        if (n >= lo) out.push_back(n);
    return out;
}

template <class T> int safe_arrays(int n, const Options& o) {  // bench.cu:600-608
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t cap = std::min(size_t(o.batchElements), free_b / (8 * sizeof(T)));
    if (cap < size_t(n)) throw std::runtime_error("Batch/memory budget cannot hold one array; increase --batch-elements");
    return int(std::min(size_t(o.arrays), cap / size_t(n)));
}

template <class T> void run_small(const Options& o, const std::string& type) {
    const int limit = b200s_max_length(dtype_of<T>(), 0);
    const int maximum = o.maxSize ? std::min(o.maxSize, limit) : reference_capacity<T>();
    if (o.minSize > maximum) return;
    Csv csv(o.prefix + "_" + type + "_small.csv", o.hbmGBs);
    for (int n : small_sizes(o.minSize, maximum)) {
        const int arrays = safe_arrays<T>(n, o);
        for (int d = 0; d < PERTURBED_32 + 1 + (o.checkOnly ? 1 : 0); ++d) {
            std::cout << "small " << type << " N=" << n << " arrays=" << arrays << ' ' << kDistNames[d] << std::endl;
            Batch<T> b(n, arrays, d, o, csv);
            small_methods(b, o);
        }
    }
}

template <class T> void run_large(const Options& o, const std::string& type) {
    const int limit = b200s_max_length(dtype_of<T>(), 0);
    const int maximum = std::min(o.maxSize ? o.maxSize : (1 << 24), limit);
    const int minimum = std::max(o.minSize, reference_capacity<T>() + 1);
    Csv csv(o.prefix + "_" + type + "_large.csv", o.hbmGBs);
    if (o.maxSize > limit)
        std::cout << "large " << type << ": lengths above " << limit << " are beyond b200sort's longest array\n";
    for (int n = working_of(minimum); n <= maximum; n *= 2) {
        for (int d = 0; d < PERTURBED_32 + 1 + (o.checkOnly ? 1 : 0); ++d) {
            std::cout << "large " << type << " N=" << n << ' ' << kDistNames[d] << std::endl;
            Batch<T> b(n, 1, d, o, csv);
            for (const std::string& m : kLarge) {
                if (!o.enabled(m.c_str())) continue;
                if (o.methods.empty() && m != "large_merge") continue;  // one row set by default
                const Config c = b200_config<T>(m, n, nullptr);
                b.run(c, [&] { return sort_b200(b, nullptr); });
            }
            if (o.enabled("thrust_segment_loop")) {
                Config c;
                c.method = "thrust_segment_loop";
                c.working = n;
                b.run(c, [&] { return thrust_segment_sort(std::is_same<T, Rec>::value ? 1 : 0, b.values.p, n, 1,
                                                          nullptr) == 0; });
            }
        }
    }
}

template <class T> void run_type(const Options& o, const std::string& type) {
    if (o.mode != "large") run_small<T>(o, type);
    if (o.mode != "small") run_large<T>(o, type);
}

}  // namespace

int main(int argc, char** argv) {
    try {
        for (int i = 1; i < argc; ++i)
            if (std::string(argv[i]) == "--help") {
                usage();
                return 0;
            }
        const Options o = parse(argc, argv);
        if (o.mode == "small" && o.maxSize) {
            if (o.type != "record" && o.maxSize > b200s_max_length(B200S_I32, 0))
                throw std::runtime_error("--max-size exceeds the longest int array (" +
                                         std::to_string(b200s_max_length(B200S_I32, 0)) + ")");
            if (o.type != "int" && o.maxSize > b200s_max_length(B200S_I32_I32, 0))
                throw std::runtime_error("--max-size exceeds the longest record array (" +
                                         std::to_string(b200s_max_length(B200S_I32_I32, 0)) + ")");
        }
        if (o.type != "record") run_type<int>(o, "int");
        if (o.type != "int") run_type<Rec>(o, "record");
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "Benchmark error: " << e.what() << '\n';
        return 1;
    }
}
