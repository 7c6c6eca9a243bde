// CPU oracle for the batched small-array sort.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker used by tests/, by the
// smoke entry and by the CPU-baseline leg of bench.py.  The product (the CUDA
// library under cuda-sort_b200/) never links, loads or calls it.
//
// It restates, on the host, what the reference (berenger-eu/cuda-sort) computes
// on its one-CTA-per-array bitonic path:
//   * per-array std::sort, which is how the reference builds its expected output
//     (bench.cu:300-301);
//   * the reflection bitonic network of cusort_v6.hpp:38-142 with the
//     keep-own-on-ties min/max of cusort.hpp:460-472, so that the exact record
//     order (including the order of records with equal keys) is predicted;
//   * the record validation of bench.cu:212-228 (key equality, payload origin in
//     range and in the same segment, input[origin] == result, uniqueness);
//   * the reference's stateless input generator (bench.cu:152-192) and its
//     locally perturbed keys (bench_distributions.hpp:11-19, bench.cu:290-297).
// Parity pin: the network restatement is checked against the reference's own
// GPU output (oracle/_ref, built from the reference headers) on the GPU box,
// and against the known-answer fixtures in tests/golden/.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

namespace {

struct Rec32 {            // layout of IntAndData (intanddata.hpp:9-11)
    int32_t val;
    int32_t data;
};
struct RecU64 {           // uint64 key + int32 payload, 16-byte AoS record
    uint64_t key;
    int32_t data;
    int32_t pad;
};

// Ordering: records compare by key only (intanddata.hpp:20-31).
inline bool less_(int32_t a, int32_t b) { return a < b; }
inline bool less_(uint64_t a, uint64_t b) { return a < b; }
inline bool less_(const Rec32& a, const Rec32& b) { return a.val < b.val; }
inline bool less_(const RecU64& a, const RecU64& b) { return a.key < b.key; }

// Padding sentinels (cusort.hpp:257-271, intanddata.hpp:47-52).
template <class T> T sentinel();
template <> int32_t sentinel<int32_t>() { return INT32_MAX; }
template <> uint64_t sentinel<uint64_t>() { return UINT64_MAX; }
template <> Rec32 sentinel<Rec32>() { return Rec32{INT32_MAX, INT32_MAX}; }
template <> RecU64 sentinel<RecU64>() { return RecU64{UINT64_MAX, INT32_MAX, 0}; }

inline int64_t working_length(int64_t n) {
    // W = next power of two >= max(32, n) (bench.cu:524, cusort_v6.hpp:133).
    int64_t w = 32;
    while (w < n) w <<= 1;
    return w;
}

// One comparator layer: element i and i ^ mask, i the lower index, i takes the
// minimum.  The exchange happens only when the upper element is strictly
// smaller, which is the reference's keep-own rule on ties
// (min(a,b) = b<a ? b : a, max(a,b) = a<b ? b : a, cusort.hpp:460-472;
// direction (index & MaximumBit) ? max : min, cusort_v6.hpp:51-56, 71, 84).
template <class T>
void layer(T* a, int64_t w, int64_t mask) {
    for (int64_t i = 0; i < w; ++i) {
        const int64_t j = i ^ mask;
        if (i < j && less_(a[j], a[i])) std::swap(a[i], a[j]);
    }
}

// The reflection bitonic network (cusort_v6.hpp:90-142): for each stage span
// S = 1, 2, ..., W/2 a reflection layer (partner i ^ (2S-1)) followed by the
// merge layers of distance S/2, ..., 1.  The reference's optional sortedness
// early exits (cusort_v6.hpp:123-125, 138-140) leave the output unchanged: a
// sorted tile is a fixed point of every layer under the keep-own rule.
template <class T>
void bitonic_one(const T* in, T* out, int64_t n, std::vector<T>& tile) {
    const int64_t w = working_length(n);
    tile.assign(size_t(w), sentinel<T>());
    std::copy(in, in + n, tile.begin());
    for (int64_t s = 1; s < w; s <<= 1) {
        layer(tile.data(), w, 2 * s - 1);
        for (int64_t d = s >> 1; d >= 1; d >>= 1) layer(tile.data(), w, d);
    }
    std::copy(tile.begin(), tile.begin() + n, out);
}

template <class F>
void parallel_for(int64_t count, int threads, F f) {
    if (threads <= 1 || count < 2) {
        for (int64_t i = 0; i < count; ++i) f(i);
        return;
    }
    std::vector<std::thread> pool;
    const int64_t chunk = (count + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int64_t lo = t * chunk, hi = std::min(count, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([lo, hi, &f] { for (int64_t i = lo; i < hi; ++i) f(i); });
    }
    for (auto& th : pool) th.join();
}

template <class T>
void sort_packed(const T* in, T* out, int64_t n, int64_t arrays, int mode, int threads) {
    parallel_for(arrays, threads, [&](int64_t a) {
        const T* src = in + a * n;
        T* dst = out + a * n;
        if (mode == 0) {                  // std::sort (bench.cu:300-301)
            std::copy(src, src + n, dst);
            std::sort(dst, dst + n, [](const T& x, const T& y) { return less_(x, y); });
        } else if (mode == 1) {           // the reference's network
            std::vector<T> tile;
            bitonic_one(src, dst, n, tile);
        } else {                          // stable: ties keep input order
            std::copy(src, src + n, dst);
            std::stable_sort(dst, dst + n, [](const T& x, const T& y) { return less_(x, y); });
        }
    });
}

template <class T>
void sort_ragged(const T* in, T* out, const int64_t* off, int64_t arrays, int mode, int threads) {
    parallel_for(arrays, threads, [&](int64_t a) {
        const int64_t lo = off[a], n = off[a + 1] - off[a];
        if (n <= 0) return;
        sort_packed(in + lo, out + lo, n, 1, mode, 1);
    });
}

inline uint32_t mix_bits(uint32_t x) {   // bench.cu:152-155
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU;
    return x ^ (x >> 16);
}

}  // namespace

extern "C" {

// dtype codes: 0 = int32 keys, 1 = int32 key + int32 payload (IntAndData),
//              2 = uint64 keys, 3 = uint64 key + int32 payload (16-byte record).
// mode: 0 = std::sort per array, 1 = the reference's bitonic network,
//       2 = std::stable_sort per array.
int orc_sort_packed(int dtype, const void* in, void* out, int64_t n, int64_t arrays,
                    int mode, int threads) {
    if (n < 0 || arrays < 0) return 1;
    if (n == 0 || arrays == 0) return 0;
    switch (dtype) {
        case 0: sort_packed((const int32_t*)in, (int32_t*)out, n, arrays, mode, threads); break;
        case 1: sort_packed((const Rec32*)in, (Rec32*)out, n, arrays, mode, threads); break;
        case 2: sort_packed((const uint64_t*)in, (uint64_t*)out, n, arrays, mode, threads); break;
        case 3: sort_packed((const RecU64*)in, (RecU64*)out, n, arrays, mode, threads); break;
        default: return 1;
    }
    return 0;
}

// Ragged batch: array a occupies [off[a], off[a+1]) of the flat buffer.
int orc_sort_ragged(int dtype, const void* in, void* out, const int64_t* off, int64_t arrays,
                    int mode, int threads) {
    switch (dtype) {
        case 0: sort_ragged((const int32_t*)in, (int32_t*)out, off, arrays, mode, threads); break;
        case 1: sort_ragged((const Rec32*)in, (Rec32*)out, off, arrays, mode, threads); break;
        case 2: sort_ragged((const uint64_t*)in, (uint64_t*)out, off, arrays, mode, threads); break;
        case 3: sort_ragged((const RecU64*)in, (RecU64*)out, off, arrays, mode, threads); break;
        default: return 1;
    }
    return 0;
}

// Record validation restated from bench.cu:204-228 for a ragged (CSR) batch;
// a packed batch is the special case off[a] = a*n.  `expected` holds keys in
// sorted order (any std::sort output).  The payload of every input record is
// its global input position, as the reference's generator sets it
// (bench.cu:189).  Returns the number of failing output positions.
int64_t orc_validate_records(const int32_t* input, const int32_t* result, const int32_t* expected,
                             const int64_t* off, int64_t arrays) {
    // input/result/expected are Rec32 viewed as int32 pairs.
    const Rec32* in = (const Rec32*)input;
    const Rec32* res = (const Rec32*)result;
    const Rec32* ref = (const Rec32*)expected;
    const int64_t count = off[arrays];
    std::vector<uint8_t> seen(static_cast<size_t>(count), 0);
    int64_t bad = 0;
    for (int64_t a = 0; a < arrays; ++a) {
        for (int64_t i = off[a]; i < off[a + 1]; ++i) {
            bool valid = !(res[i].val < ref[i].val) && !(ref[i].val < res[i].val);
            const int64_t origin = res[i].data;
            if (origin < off[a] || origin >= off[a + 1]) valid = false;
            else {
                if (in[origin].val != res[i].val || in[origin].data != res[i].data) valid = false;
                if (seen[size_t(origin)]++) valid = false;
            }
            if (!valid) ++bad;
        }
    }
    return bad;
}

uint32_t orc_mix_bits(uint32_t x) { return mix_bits(x); }

// The reference's stateless batch initialiser (bench.cu:159-192), restated on
// the host for int32 keys (dtype 0) or IntAndData records (dtype 1, payload =
// global index).  distribution: 0 SORTED, 1 REVERSED, 2 RANDOM, 3 NORMAL,
// 4 CONSTANT, 5 BINARY (valgen.hpp:7-15), 6/7/8 PERTURBED_2/8/32
// (bench.cu:26-31, keys then perturbed as bench.cu:290-297), 9 EXTREMES.
// NORMAL uses the host libm; the reference evaluates it on the device, so a
// rare key may differ by one.  No parity claim rests on NORMAL inputs.
int orc_ref_initialize(int dtype, void* data, int64_t n, int64_t arrays, int distribution) {
    const int64_t count = n * arrays;
    if (n <= 0 || count > INT32_MAX) return 1;
    std::vector<int32_t> keys(static_cast<size_t>(count));
    for (int64_t i = 0; i < count; ++i) {
        const int64_t local = i % n;
        const uint32_t random = mix_bits(uint32_t(i) + 1234U);
        int32_t key = 0;
        switch (distribution) {
            case 0: case 6: case 7: case 8: key = int32_t(local); break;
            case 1: key = int32_t(n - 1 - local); break;
            case 2: key = int32_t(random % 1000001U); break;
            case 3: {
                const float u = (float(random & 0xffffffU) + 1.0f) / 16777217.0f;
                const float v = float(mix_bits(random) & 0xffffffU) / 16777216.0f;
                const float z = std::sqrt(-2.0f * std::log(u)) * std::cos(6.28318530718f * v);
                key = int32_t(z * (1.0f + float(n) / 4.0f) + float(n) / 2.0f);
                key = key < 0 ? 0 : (key > n ? int32_t(n) : key);
                break;
            }
            case 4: key = 99; break;
            case 5: key = int32_t(local % 2); break;
            default: {
                static const int32_t extremes[] = {INT32_MAX, INT32_MIN, 0, INT32_MAX, -1, 1};
                key = extremes[local % 6];
            }
        }
        keys[size_t(i)] = key;
    }
    int amplitude = 0;
    if (distribution == 6) amplitude = 2;
    if (distribution == 7) amplitude = 8;
    if (distribution == 8) amplitude = 32;
    if (amplitude) {
        // generateLocallyPerturbedKeys: x[i] = 4i + U{-4r..4r}, mt19937(seed)
        // with seed = mixBits(a + 1234) (bench_distributions.hpp:11-19).
        for (int64_t a = 0; a < arrays; ++a) {
            std::mt19937 rng(mix_bits(uint32_t(a) + 1234U));
            const int delta = 4 * amplitude;
            std::uniform_int_distribution<int> noise(-delta, delta);
            for (int64_t i = 0; i < n; ++i) keys[size_t(a * n + i)] = int32_t(4 * i + noise(rng));
        }
    }
    if (dtype == 0) {
        std::memcpy(data, keys.data(), size_t(count) * 4);
    } else if (dtype == 1) {
        Rec32* r = (Rec32*)data;
        for (int64_t i = 0; i < count; ++i) r[i] = Rec32{keys[size_t(i)], int32_t(i)};
    } else {
        return 1;
    }
    return 0;
}

}  // extern "C"
