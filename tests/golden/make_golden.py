"""Generate the known-answer fixtures in tests/golden/kat.json.

Pure Python, independent of the C++ oracle, so that the two restatements
check each other.  The cases are the reference's own known-answer inputs for
the small-array path: the EXTREMES cycle {INT_MAX, INT_MIN, 0, INT_MAX, -1, 1}
(bench.cu:184-187), CONSTANT = 99 (bench.cu:182), SORTED / REVERSED
(bench.cu:167-171), BINARY (bench.cu:183) and RANDOM = mixBits(i + 1234) %
1000001 (bench.cu:172), at the edge lengths of the reference's size sweep
(1..33, 2^k - 1, 2^k, 2^k + 1; bench.cu:587-598).  Records carry payload =
global index (bench.cu:189).  Expected outputs: the sorted key sequence
(what the reference compares against, bench.cu:300-301) and, for records, the
full record order produced by the reference's comparator network
(cusort_v6.hpp:38-142 with the keep-own tie rule of cusort.hpp:460-472).

Run: python tests/golden/make_golden.py   (rewrites kat.json)
"""
import json
import os

INT_MAX = 2**31 - 1
INT_MIN = -2**31


def mix_bits(x):
    x &= 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    return x ^ (x >> 16)


def ref_keys(dist, n, arrays):
    out = []
    for i in range(n * arrays):
        local = i % n
        if dist == "SORTED":
            k = local
        elif dist == "REVERSED":
            k = n - 1 - local
        elif dist == "RANDOM":
            k = mix_bits(i + 1234) % 1000001
        elif dist == "CONSTANT":
            k = 99
        elif dist == "BINARY":
            k = local % 2
        else:
            k = [INT_MAX, INT_MIN, 0, INT_MAX, -1, 1][local % 6]
        out.append(k)
    return out


def network(recs):
    """Reflection bitonic network over W = next pow2 >= max(32, n)."""
    n = len(recs)
    w = 32
    while w < n:
        w *= 2
    a = list(recs) + [(INT_MAX, INT_MAX)] * (w - n)
    s = 1
    while s < w:
        masks = [2 * s - 1]
        d = s // 2
        while d >= 1:
            masks.append(d)
            d //= 2
        for m in masks:
            for i in range(w):
                j = i ^ m
                if i < j and a[j][0] < a[i][0]:
                    a[i], a[j] = a[j], a[i]
        s *= 2
    return a[:n]


def main():
    lengths = sorted(set(list(range(1, 34)) + [63, 64, 65, 127, 128, 129, 255, 256, 257]))
    cases = []
    for dist in ("EXTREMES", "CONSTANT", "SORTED", "REVERSED", "BINARY", "RANDOM"):
        for n in lengths:
            arrays = 2
            keys = ref_keys(dist, n, arrays)
            recs = [(k, i) for i, k in enumerate(keys)]
            exp_keys, exp_recs = [], []
            for a in range(arrays):
                seg = recs[a * n:(a + 1) * n]
                exp_keys += sorted(k for k, _ in seg)
                exp_recs += network(seg)
            cases.append({"distribution": dist, "n": n, "arrays": arrays, "keys": keys,
                          "sorted_keys": exp_keys, "network_records": [list(r) for r in exp_recs]})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat.json")
    with open(path, "w") as f:
        json.dump({"cases": cases}, f, separators=(",", ":"))
    print("wrote", path, len(cases), "cases")


if __name__ == "__main__":
    main()
