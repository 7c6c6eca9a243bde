"""Inputs of the reference-output fixture (tests/golden/ref_network.json).

A self-contained generator (splitmix64 over the global element index, in
numpy uint64 arithmetic) so that the GPU script that records the reference's
output and the CPU test that checks the oracle against it build bit-identical
inputs on any machine, independent of numpy's random-stream versions.
Records are IntAndData {int32 key; int32 data} with data = global index, as
the reference's generator sets it (bench.cu:189).  Every distribution is
chosen for ties, which is where record order depends on the network:
  distinct16  keys from 16 values spread over the int32 range
  equal       one key for the whole batch
  near3       nearly sorted, about three records per key: (i + r%9 - 4) // 3
  extremes    keys from {INT32_MIN, -1, 0, 1, 5, INT32_MAX} (INT32_MAX ties
              the padding key, which must never enter the valid prefix)
"""
import numpy as np

DISTRIBUTIONS = ("distinct16", "equal", "near3", "extremes")
REC = np.dtype([("key", "<i4"), ("data", "<i4")])


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def records(n, arrays, dist, seed):
    """A packed batch of `arrays` x n records."""
    total = n * arrays
    i = np.arange(total, dtype=np.uint64)
    r = splitmix64(i ^ (np.uint64(seed) << np.uint64(32)))
    pos = (np.arange(total, dtype=np.int64) % max(n, 1))
    if dist == "distinct16":
        keys = -2147483648 + (r % np.uint64(16)).astype(np.int64) * 286331153
    elif dist == "equal":
        keys = np.full(total, 42, dtype=np.int64)
    elif dist == "near3":
        keys = (pos + (r % np.uint64(9)).astype(np.int64) - 4) // 3
    elif dist == "extremes":
        vals = np.array([-2147483648, -1, 0, 1, 5, 2147483647], dtype=np.int64)
        keys = vals[(r % np.uint64(6)).astype(np.int64)]
    else:
        raise ValueError(dist)
    out = np.empty(total, dtype=REC)
    out["key"] = keys.astype(np.int32)
    out["data"] = np.arange(total, dtype=np.int32)
    return out


def cases():
    """(n, arrays, dist, seed, threads, sorted) of every fixture case; threads
    is the reference V6 block size (working / threads <= 16, bench.cu:497-521)."""
    out = []
    for n in (1, 2, 3, 16, 31, 32, 33, 64, 100, 129, 255, 256, 500, 1000, 1024, 1500, 2048):
        w = 32
        while w < n:
            w *= 2
        arrays = 3 if n <= 256 else 1
        for k, dist in enumerate(DISTRIBUTIONS):
            seed = n * 8 + k
            out.append((n, arrays, dist, seed, max(32, w // 16), 0))
            if dist == "near3":
                # the reference's Sorted switch (early exits) on the same input
                out.append((n, arrays, dist, seed, max(32, w // 4), 1))
    return out
