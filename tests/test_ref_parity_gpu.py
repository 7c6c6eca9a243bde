"""GPU parity against the reference itself: its V6 / V4 / V3 / V2 / V1 / warp kernels,
compiled unmodified from its headers for sm_100a (oracle/_ref), run on the
same inputs as the new kernels and the CPU oracle.  Records with many equal
keys make the comparison cover the tie order, not only the keys."""
import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.ref_gpu_available(), reason="reference GPU kernels not built")]

CAP = {bs.I32: 4096, bs.I32_I32: 2048}   # the reference's small-path capacity (cusort.hpp:231-237)


def working(n):
    w = 32
    while w < n:
        w *= 2
    return w


def run_ref(kind, dtype, data, n, arrays, threads=None, sorted_=0, shared=0, async_=0):
    import torch
    suffix = "int" if dtype == bs.I32 else "rec"
    lib = orc.ref_gpu(suffix)
    d = to_device(data)
    w = working(n)
    st = stream_handle()
    if kind == "v6":
        rc = getattr(lib, "ref_v6_" + suffix)(d.data_ptr(), n, arrays, w, threads, sorted_, shared, async_, st)
    elif kind == "v4":
        rc = getattr(lib, "ref_v4_" + suffix)(d.data_ptr(), n, arrays, w, threads, sorted_, shared, async_, st)
    elif kind == "v3":
        rc = getattr(lib, "ref_v3_" + suffix)(d.data_ptr(), n, arrays, w, threads, sorted_, shared, async_, st)
    elif kind in ("v1", "v2"):
        rc = getattr(lib, "ref_v12_" + suffix)(d.data_ptr(), n, arrays, int(kind[1]), w, sorted_, shared, st)
    else:
        rc = getattr(lib, "ref_warp_" + suffix)(d.data_ptr(), n, arrays, sorted_, shared, st)
    assert rc == 0, (kind, n, threads, rc)
    torch.cuda.synchronize()
    return from_device(d[:data.nbytes], bs.NP_DTYPES[dtype])


def run_ours(dtype, data, n, arrays):
    import torch
    d_in = to_device(data)
    d_out = empty_device(d_in.numel())
    bs.sort_packed(dtype, d_in.data_ptr(), d_out.data_ptr(), n, arrays, 0, None, stream_handle())
    torch.cuda.synchronize()
    return from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype])


INPUTS = [("distinct16", True), ("equal", False), ("swap8", True), ("uniform", True), ("organ", False)]


@pytest.mark.parametrize("dtype", [bs.I32, bs.I32_I32])
def test_v6_equals_oracle_and_new_kernels(dtype):
    for n in (1, 2, 17, 31, 32, 33, 100, 129, 255, 256, 513, 1000, 1024, 1025, 2000, 2048, 3000, 4096):
        if n > CAP[dtype]:
            continue
        w = working(n)
        for dist, ext in INPUTS:
            arrays = 6
            data = workloads.make_packed(dtype, n, arrays, dist, seed=n + 11, extremes=ext)
            net = orc.sort_packed(dtype, data, n, arrays, orc.MODE_NETWORK)
            ours = run_ours(dtype, data, n, arrays)
            assert np.array_equal(ours, net), (n, dist)
            for threads in sorted({max(32, w // 16), min(w, 128), min(w, 1024)}):
                if w // threads > 16 or threads > w:
                    continue
                ref = run_ref("v6", dtype, data, n, arrays, threads)
                assert np.array_equal(ref, net), ("v6", n, threads, dist)


@pytest.mark.parametrize("dtype", [bs.I32, bs.I32_I32])
def test_reference_variants_share_one_network(dtype):
    # Sorted / Shared / Async switches and the V3, V4 and warp kernels all
    # produce the record order of the same comparator network.
    for n in (5, 32, 33, 200, 1024, 2048):
        w = working(n)
        data = workloads.make_packed(dtype, n, 4, "distinct16", seed=n, extremes=True)
        net = orc.sort_packed(dtype, data, n, 4, orc.MODE_NETWORK)
        threads = min(w, 256) if w // min(w, 256) <= 16 else w // 16
        for s, sh, a in ((1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1)):
            assert np.array_equal(run_ref("v6", dtype, data, n, 4, threads, s, sh, a), net), (n, s, sh, a)
        if n >= 32:
            for s, sh, a in ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)):
                t = min(w, 256)
                assert np.array_equal(run_ref("v4", dtype, data, n, 4, t, s, sh, a), net), ("v4", n)
                assert np.array_equal(run_ref("v3", dtype, data, n, 4, t, s, sh, a), net), ("v3", n)
        else:
            for s, sh in ((0, 0), (1, 0), (0, 1), (1, 1)):
                assert np.array_equal(run_ref("warp", dtype, data, n, 4, None, s, sh), net), ("warp", n)


def test_reference_inputs_full_batch_records():
    # The reference's own generator and sizes: EXTREMES and PERTURBED cases.
    for dist in ("EXTREMES", "PERTURBED_8", "BINARY", "RANDOM"):
        for n in (129, 1000, 2048):
            arrays = 2048
            data = orc.ref_initialize(1, n, arrays, dist, bs.NP_DTYPES[bs.I32_I32])
            w = working(n)
            ref = run_ref("v6", bs.I32_I32, data, n, arrays, max(32, w // 8))
            ours = run_ours(bs.I32_I32, data, n, arrays)
            assert np.array_equal(ours, ref), (dist, n)


@pytest.mark.parametrize("kind", ["v1", "v2"])
@pytest.mark.parametrize("dtype", [bs.I32, bs.I32_I32])
def test_v1_v2_equal_oracle_and_new_kernels(kind, dtype):
    # one value per thread, the whole array in one block of `working` threads
    # (cusort.hpp:751-771, 986-1008): every length up to 1024
    for n in (1, 2, 17, 31, 32, 33, 100, 129, 255, 256, 500, 512, 513, 1000, 1024):
        arrays = 5
        for dist, extremes in INPUTS:
            data = workloads.make_packed(dtype, n, arrays, dist, seed=n + 3, extremes=extremes)
            oracle = orc.sort_packed(dtype, data, n, arrays, orc.MODE_NETWORK if dtype else orc.MODE_STD)
            for sorted_, shared in ((0, 0), (1, 0), (0, 1), (1, 1)):
                ref = run_ref(kind, dtype, data, n, arrays, sorted_=sorted_, shared=shared)
                assert np.array_equal(ref, oracle), (kind, dtype, n, dist, sorted_, shared)
            assert np.array_equal(run_ours(dtype, data, n, arrays), oracle), (dtype, n, dist)
