"""The allocation-free ragged sort (b200s_sort_ragged_noalloc) against the
plan-based one (b200s_sort_ragged).

Callers that cannot allocate device memory — plugins inside a framework that
owns all device memory through its own pool, latency-critical loops that
cannot afford cudaMalloc's device-wide synchronisation — use the entry point
whose scratch is a fixed array compiled into the library.  Its output must be
the plan path's output, bit for bit, on consecutive calls (the shared scratch
keeps the previous call's contents), and a batch larger than its fixed
capacity must be rejected with a clear error.  This file is collected last so
that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import b200sort as bs
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device

pytestmark = pytest.mark.gpu

MAX_ARRAYS = 32768   # B200S_NOALLOC_MAX_ARRAYS in include/b200sort.h


def _noalloc():
    return bs.declare("b200s_sort_ragged_noalloc", ctypes.c_int,
                      [ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_int64, ctypes.c_void_p])


def _batch(dtype, arrays, max_len, seed):
    lengths = workloads.ragged_lengths(arrays, max_len=max_len, seed=seed)
    lengths[::53] = 0
    return workloads.make_ragged(dtype, lengths, "distinct16", seed=seed, extremes=True)


def _run_both(dtype, flags, data, off):
    import torch
    st = stream_handle()
    d_in = to_device(data)
    d_off = torch.from_numpy(off.astype(np.int32)).cuda()
    out_plan = empty_device(d_in.numel())
    out_free = empty_device(d_in.numel())
    arrays = len(off) - 1
    with bs.Plan(dtype, arrays, flags) as plan:
        plan.sort(d_in.data_ptr(), out_plan.data_ptr(), d_off.data_ptr(), arrays, st)
    rc = _noalloc()(dtype, flags, d_in.data_ptr(), out_free.data_ptr(), d_off.data_ptr(), arrays, st)
    assert rc == 0, bs.lib().b200s_last_error().decode()
    torch.cuda.synchronize()
    npd = bs.NP_DTYPES[dtype]
    return from_device(out_plan[:data.nbytes], npd), from_device(out_free[:data.nbytes], npd)


@pytest.mark.parametrize("dtype,flags", [(bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.I32, 0),
                                         (bs.U64_I32, 0)])
def test_noalloc_matches_plan_on_two_calls_in_a_row(dtype, flags):
    top = bs.ragged_max_length(dtype, flags)
    # first call: many short arrays plus a few long enough for the cluster kernels
    data1, off1 = _batch(dtype, 3000, min(top, 20000), seed=101)
    plan1, free1 = _run_both(dtype, flags, data1, off1)
    assert np.array_equal(free1, plan1)
    # second call: a different batch; the scratch still holds the first call's state
    data2, off2 = _batch(dtype, 700, 2048, seed=202)
    plan2, free2 = _run_both(dtype, flags, data2, off2)
    assert np.array_equal(free2, plan2)


@pytest.mark.parametrize("dtype", [bs.I32_I32, bs.U64_I32])
def test_noalloc_long_arrays_take_the_plans_cluster_tiles(dtype):
    # arrays of 16385 .. 65536 records reach the largest cluster buckets; both
    # paths must run the same tile there, so outputs (tie order included)
    # match and the no-alloc call is not slower than the plan's
    top = bs.ragged_max_length(dtype, 0)
    assert top >= 65536
    rng = np.random.default_rng(303)
    lengths = np.concatenate([rng.integers(32769, 65537, size=6), rng.integers(16385, 32769, size=4),
                              rng.integers(1, 3000, size=40)])
    rng.shuffle(lengths)
    data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=303, extremes=True)
    for _ in range(2):
        plan, free = _run_both(dtype, 0, data, off)
        assert np.array_equal(free, plan)


def test_noalloc_rejects_batches_beyond_its_capacity():
    fn = _noalloc()
    rc = fn(bs.I32, 0, 16, 16, 16, MAX_ARRAYS + 1, 0)
    assert rc == 1
    assert str(MAX_ARRAYS) in bs.lib().b200s_last_error().decode()
    assert fn(bs.I32, 0, 16, 16, 16, 0, 0) == 0
