"""Seeded synthetic batches for the benchmark and the tests (host side, numpy).

Distributions (every array is generated independently from the seed):
  uniform     i.i.d. keys over the full key range
  sorted      uniform keys sorted ascending
  reverse     uniform keys sorted descending
  equal       one key value for the whole array
  distinct16  keys drawn from 16 values spread over the key range
  organ       organ pipe: min(i, n-1-i)
  swap1/swap8/swap64
              sorted keys, then bounded random swaps: each swap exchanges two
              positions at most r apart (r = 1, 8, 64), in non-overlapping
              windows of 2r positions, two rounds offset by r
With `extremes=True` every array of length >= 2 also receives the minimum and
the maximum key at seeded positions, and arrays of length >= 4 a duplicated
key, so every batch exercises the padding and tie rules.

Record payloads are the global input position of the record, as the
reference's generator sets them (bench.cu:189); the record validator relies
on that to check that each payload stays with its key and its array.
"""
import numpy as np

from b200sort import I32, I32_I32, U64, U64_I32, NP_DTYPES

DISTRIBUTIONS = ("uniform", "sorted", "reverse", "equal", "distinct16", "organ",
                 "swap1", "swap8", "swap64")


def _key_info(dtype):
    if dtype in (I32, I32_I32):
        return np.int32, np.iinfo(np.int32)
    return np.uint64, np.iinfo(np.uint64)


def _uniform(rng, shape, dtype):
    kt, info = _key_info(dtype)
    if kt == np.int32:
        return rng.integers(info.min, info.max, size=shape, dtype=np.int64, endpoint=True).astype(np.int32)
    return rng.integers(0, np.iinfo(np.uint64).max, size=shape, dtype=np.uint64, endpoint=True)


def _swaps(keys, r, rng):
    arrays, n = keys.shape
    rows = np.arange(arrays)[:, None]
    for off in (0, r):
        nw = (n - off) // (2 * r)
        if nw <= 0:
            continue
        u = rng.integers(0, r, size=(arrays, nw))
        d = rng.integers(1, r + 1, size=(arrays, nw))
        coin = rng.random((arrays, nw)) < 0.5
        i = off + np.arange(nw)[None, :] * 2 * r + u
        j = i + d
        ii = np.where(coin, i, j)
        a, b = keys[rows, ii].copy(), keys[rows, j].copy()
        keys[rows, ii] = b
        keys[rows, j] = a
    return keys


def keys_2d(dtype, n, arrays, distribution, rng):
    """Keys of shape (arrays, n) for one of DISTRIBUTIONS."""
    kt, info = _key_info(dtype)
    if distribution == "uniform":
        return _uniform(rng, (arrays, n), dtype)
    if distribution in ("sorted", "reverse") or distribution.startswith("swap"):
        k = np.sort(_uniform(rng, (arrays, n), dtype), axis=1)
        if distribution == "reverse":
            k = k[:, ::-1].copy()
        elif distribution.startswith("swap"):
            k = _swaps(k, int(distribution[4:]), rng)
        return k
    if distribution == "equal":
        return np.full((arrays, n), 42, dtype=kt)
    if distribution == "distinct16":
        vals = np.linspace(float(info.min), float(info.max), 16)
        vals = np.array([int(v) for v in vals], dtype=object)
        vals = np.clip(vals, int(info.min), int(info.max)).astype(kt)
        return vals[rng.integers(0, 16, size=(arrays, n))]
    if distribution == "organ":
        i = np.arange(n)
        return np.broadcast_to(np.minimum(i, n - 1 - i).astype(kt), (arrays, n)).copy()
    raise ValueError("unknown distribution %r" % distribution)


def inject_extremes(keys, dtype, rng):
    """Place the minimum and maximum key and one duplicate in every array."""
    arrays, n = keys.shape
    if n < 2 or arrays == 0:
        return keys
    kt, info = _key_info(dtype)
    rows = np.arange(arrays)
    p = np.argsort(rng.random((arrays, n)), axis=1)[:, :4] if n >= 4 else \
        np.argsort(rng.random((arrays, n)), axis=1)
    keys[rows, p[:, 0]] = kt(info.min)
    keys[rows, p[:, 1]] = kt(info.max)
    if n >= 4:
        keys[rows, p[:, 3]] = keys[rows, p[:, 2]]
    return keys


def make_packed(dtype, n, arrays, distribution="uniform", seed=1234, extremes=False):
    """A packed batch (arrays * n elements) as a 1-D numpy array of NP_DTYPES[dtype]."""
    rng = np.random.default_rng(seed)
    keys = keys_2d(dtype, n, arrays, distribution, rng)
    if extremes:
        keys = inject_extremes(keys, dtype, rng)
    return _assemble(dtype, keys.reshape(-1))


def _assemble(dtype, flat_keys):
    out = np.empty(flat_keys.shape[0], dtype=NP_DTYPES[dtype])
    if dtype in (I32, U64):
        out[:] = flat_keys
    else:
        out["key"] = flat_keys
        out["data"] = np.arange(flat_keys.shape[0], dtype=np.int64).astype(np.int32)
        if dtype == U64_I32:
            out["reserved"] = 0
    return out


def ragged_lengths(arrays, max_len=8192, seed=1234, min_len=1):
    """Lengths floor(exp(U * ln(max_len))), log-uniform on [1, max_len], then
    clamped to [min_len, max_len]."""
    rng = np.random.default_rng(seed)
    u = rng.random(arrays)
    lens = np.floor(np.exp(u * np.log(max_len))).astype(np.int64)
    return np.clip(lens, min_len, max_len)


def log_uniform_lengths(count, lo, hi, seed=1234):
    """Lengths log-uniform on [lo, hi]: floor(exp(ln lo + U * (ln hi - ln lo)))."""
    rng = np.random.default_rng(seed)
    u = rng.random(count)
    lens = np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)
    return np.clip(lens, lo, hi)


def offsets_from_lengths(lengths):
    off = np.zeros(len(lengths) + 1, dtype=np.int64)
    np.cumsum(lengths, out=off[1:])
    return off


def make_ragged(dtype, lengths, distribution="uniform", seed=1234, extremes=False):
    """A ragged batch: flat elements and CSR offsets (int64, arrays + 1)."""
    rng = np.random.default_rng(seed)
    off = offsets_from_lengths(lengths)
    total = int(off[-1])
    if distribution == "uniform" and not extremes:
        keys = _uniform(rng, (total,), dtype)
    else:
        keys = np.empty(total, dtype=_key_info(dtype)[0])
        for n in np.unique(lengths):
            ids = np.nonzero(lengths == n)[0]
            k = keys_2d(dtype, int(n), len(ids), distribution, rng)
            if extremes:
                k = inject_extremes(k, dtype, rng)
            idx = off[ids][:, None] + np.arange(int(n))[None, :]
            keys[idx.reshape(-1)] = k.reshape(-1)
    return _assemble(dtype, keys), off
