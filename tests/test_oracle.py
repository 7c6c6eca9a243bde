"""CPU checks of the oracle: known answers, the network restatement, the record
validator, and the reference's CPU path when it was built here."""
import json
import os

import numpy as np
import pytest

import cpu_oracle as orc
import workloads
from b200sort import I32, I32_I32, U64, U64_I32, NP_DTYPES

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REC = NP_DTYPES[I32_I32]


def _records(keys):
    r = np.empty(len(keys), dtype=REC)
    r["key"] = np.asarray(keys, dtype=np.int64).astype(np.int32)
    r["data"] = np.arange(len(keys), dtype=np.int32)
    return r


def _py_network(recs, w):
    """Reflection network over an explicit working length w >= len(recs)."""
    n = len(recs)
    a = list(recs) + [(2**31 - 1, 2**31 - 1)] * (w - n)
    s = 1
    while s < w:
        masks = [2 * s - 1] + [s >> k for k in range(1, s.bit_length())]
        for m in masks:
            for i in range(w):
                j = i ^ m
                if i < j and a[j][0] < a[i][0]:
                    a[i], a[j] = a[j], a[i]
        s *= 2
    return a[:n]


def test_known_answers_from_the_reference_inputs():
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        cases = json.load(f)["cases"]
    assert len(cases) >= 200
    for c in cases:
        n, arrays = c["n"], c["arrays"]
        keys = np.array(c["keys"], dtype=np.int64).astype(np.int32)
        got = orc.sort_packed(I32, keys, n, arrays, orc.MODE_STD)
        assert got.tolist() == c["sorted_keys"], (c["distribution"], n)
        got = orc.sort_packed(I32, keys, n, arrays, orc.MODE_NETWORK)
        assert got.tolist() == c["sorted_keys"], (c["distribution"], n)
        recs = _records(keys)
        net = orc.sort_packed(I32_I32, recs, n, arrays, orc.MODE_NETWORK)
        assert [[int(k), int(d)] for k, d in zip(net["key"], net["data"])] == c["network_records"], \
            (c["distribution"], n)


def test_reference_generator_restatement_matches_fixture_inputs():
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        cases = json.load(f)["cases"]
    for c in cases[:120]:
        got = orc.ref_initialize(0, c["n"], c["arrays"], c["distribution"], np.int32)
        assert got.tolist() == c["keys"], (c["distribution"], c["n"])
    assert orc.mix_bits(0) == 0
    assert orc.mix_bits(1234) != 1234


@pytest.mark.parametrize("n", [1, 2, 5, 17, 32, 33, 100, 128, 257, 1000, 1024, 2049, 4096])
@pytest.mark.parametrize("dist", workloads.DISTRIBUTIONS)
def test_network_keys_equal_std_sort(n, dist):
    for dtype in (I32, I32_I32, U64, U64_I32):
        data = workloads.make_packed(dtype, n, 3, dist, seed=n * 7 + 1, extremes=True)
        std = orc.sort_packed(dtype, data, n, 3, orc.MODE_STD)
        net = orc.sort_packed(dtype, data, n, 3, orc.MODE_NETWORK)
        stab = orc.sort_packed(dtype, data, n, 3, orc.MODE_STABLE)
        if dtype in (I32, U64):
            assert np.array_equal(std, net) and np.array_equal(std, stab)
        else:
            assert np.array_equal(std["key"], net["key"])
            assert np.array_equal(std["key"], stab["key"])


@pytest.mark.parametrize("n", [1, 3, 9, 16, 31, 40, 64, 100])
def test_network_output_does_not_depend_on_working_length(n):
    # Padding with the maximum key never moves under the keep-own rule, so
    # every power-of-two W >= n gives the same record order.  The kernels
    # rely on this to pick W per tile.
    rng = np.random.default_rng(n)
    keys = rng.integers(-3, 3, size=n)
    keys[rng.integers(0, n)] = 2**31 - 1
    recs = [(int(k), i) for i, k in enumerate(keys)]
    w0 = 1
    while w0 < n:
        w0 *= 2
    ref = _py_network(recs, max(32, w0))
    for w in (w0, 2 * w0, 4 * w0):
        assert _py_network(recs, w) == ref
    got = orc.sort_packed(I32_I32, _records(keys), n, 1, orc.MODE_NETWORK)
    assert [(int(k), int(d)) for k, d in zip(got["key"], got["data"])] == ref


def test_network_is_not_stable_but_stable_mode_is():
    keys = np.array([5, 5, 1, 5, 1, 1, 5, 0] * 8, dtype=np.int32)
    recs = _records(keys)
    net = orc.sort_packed(I32_I32, recs, len(keys), 1, orc.MODE_NETWORK)
    stab = orc.sort_packed(I32_I32, recs, len(keys), 1, orc.MODE_STABLE)
    expect = sorted(range(len(keys)), key=lambda i: (keys[i], i))
    assert stab["data"].tolist() == expect
    assert net["key"].tolist() == stab["key"].tolist()
    assert net["data"].tolist() != stab["data"].tolist()


def test_record_validator_accepts_correct_and_catches_planted_mistakes():
    n, arrays = 64, 4
    data = workloads.make_packed(I32_I32, n, arrays, "distinct16", seed=3, extremes=True)
    off = np.arange(arrays + 1, dtype=np.int64) * n
    expected = orc.sort_packed(I32_I32, data, n, arrays, orc.MODE_STD)
    good = orc.sort_packed(I32_I32, data, n, arrays, orc.MODE_NETWORK)
    assert orc.validate_records(data, good, expected, off) == 0
    # payload moved to another array
    bad = good.copy()
    bad["data"][0], bad["data"][n] = bad["data"][n], bad["data"][0]
    assert orc.validate_records(data, bad, expected, off) > 0
    # a record duplicated over another
    bad = good.copy()
    bad[5] = bad[6]
    assert orc.validate_records(data, bad, expected, off) > 0
    # a key changed
    bad = good.copy()
    bad["key"][7] ^= 1
    assert orc.validate_records(data, bad, expected, off) > 0
    # the padding record leaking into the output
    bad = good.copy()
    bad[n - 1] = (2**31 - 1, 2**31 - 1)
    assert orc.validate_records(data, bad, expected, off) > 0


def test_ragged_oracle_matches_packed():
    lengths = workloads.ragged_lengths(300, max_len=600, seed=5)
    data, off = workloads.make_ragged(I32_I32, lengths, "uniform", seed=6, extremes=True)
    out = orc.sort_ragged(I32_I32, data, off, orc.MODE_NETWORK, threads=4)
    for a in range(0, 300, 37):
        lo, hi = off[a], off[a + 1]
        seg = orc.sort_packed(I32_I32, data[lo:hi], hi - lo, 1, orc.MODE_NETWORK)
        assert np.array_equal(out[lo:hi], seg)
    expected = orc.sort_ragged(I32_I32, data, off, orc.MODE_STD, threads=4)
    assert orc.validate_records(data, out, expected, off) == 0


def test_reference_perturbed_keys_stay_in_their_band():
    n, arrays = 500, 3
    for dist, r in (("PERTURBED_2", 2), ("PERTURBED_8", 8), ("PERTURBED_32", 32)):
        k = orc.ref_initialize(0, n, arrays, dist, np.int32).reshape(arrays, n)
        base = 4 * np.arange(n)
        assert np.all(np.abs(k - base) <= 4 * r)
        assert not np.array_equal(k[0], k[1])


@pytest.mark.skipif(not orc.ref_cpu_available(), reason="reference CPU path not built here")
def test_reference_cpu_sort_keys_equal_oracle():
    for type_code, dtype in ((0, I32), (1, I32_I32)):
        for n in (1, 33, 1000):
            data = workloads.make_packed(dtype, n, 5, "distinct16", seed=n, extremes=True)
            ref = data.copy()
            orc.ref_cpu_sort_inplace(type_code, ref, n, 5, 2)
            std = orc.sort_packed(dtype, data, n, 5, orc.MODE_STD)
            if dtype == I32:
                assert np.array_equal(ref, std)
            else:
                assert np.array_equal(ref["key"], std["key"])
                off = np.arange(6, dtype=np.int64) * n
                assert orc.validate_records(data, ref, std, off) == 0
