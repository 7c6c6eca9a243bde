"""GPU parity of the TMA-pipelined launch form (b200s_tile.persistent = 2):
every tile that has it, against the oracle, over chunk-boundary batch sizes,
padded lengths, in place and out of place, and the fallback to the one-shot
kernel for batches that do not meet its row alignment."""
import ctypes

import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device

pytestmark = pytest.mark.gpu

# (dtype, log2_items, log2_lanes) of the tiles compiled with the TMA form
TMA_TILES = [(bs.I32, 5, 5), (bs.I32, 5, 4), (bs.I32, 4, 5), (bs.I32, 5, 3), (bs.I32, 5, 2), (bs.I32, 5, 0),
             (bs.I32_I32, 4, 1), (bs.I32_I32, 4, 2), (bs.I32_I32, 4, 3), (bs.I32_I32, 4, 4), (bs.I32_I32, 4, 5),
             (bs.I32_I32, 5, 5)]


def expected(dtype, data, n, arrays):
    mode = orc.MODE_STD if dtype in (bs.I32, bs.U64) else orc.MODE_NETWORK
    return orc.sort_packed(dtype, data, n, arrays, mode, threads=16)


def sort_with(dtype, tile, data, n, arrays, inplace):
    import torch
    d_in = to_device(data)
    d_out = d_in if inplace else empty_device(d_in.numel())
    bs.sort_packed(dtype, d_in.data_ptr(), d_out.data_ptr(), n, arrays, 0, tile, stream_handle())
    torch.cuda.synchronize()
    return from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype])


def timeouts():
    c = ctypes.c_int64(-1)
    fn = bs.declare("b200s_tma_timeouts", ctypes.c_int, [ctypes.POINTER(ctypes.c_int64)])
    assert fn(ctypes.byref(c)) == 0
    return c.value


@pytest.mark.parametrize("dtype,lk,lg", TMA_TILES)
def test_tma_form_matches_oracle(dtype, lk, lg):
    t0 = timeouts()
    eb = bs.ELEM_BYTES[dtype]
    w = 1 << (lk + lg)
    row = 128 // eb                       # elements per 128-byte row
    tpa = 1 << lg
    apc = 128 // tpa                      # arrays per CTA chunk
    lengths = sorted({w, max(row, w - row), max(row, w // 2 // row * row)})
    tile = bs.Tile(lk, lg, 0, 0, 2, 0)
    for n in lengths:
        if n % row or n > w:
            continue
        for arrays in (1, apc - 1 if apc > 1 else 1, apc + 1, 3 * apc + 5, 2000):
            for dist in ("distinct16", "uniform"):
                data = workloads.make_packed(dtype, n, arrays, dist, seed=n * 7 + arrays, extremes=True)
                want = expected(dtype, data, n, arrays)
                for inplace in (False, True):
                    got = sort_with(dtype, tile, data, n, arrays, inplace)
                    assert np.array_equal(got, want), "tile K=%d G=%d n=%d arrays=%d %s inplace=%s" % (
                        1 << lk, tpa, n, arrays, dist, inplace)
    assert timeouts() == t0


def test_tma_form_large_batches_every_distribution():
    t0 = timeouts()
    for dtype, n, arrays in ((bs.I32, 1024, 4096), (bs.I32_I32, 32, 131072), (bs.I32_I32, 256, 16384)):
        t = bs.default_tile(dtype, n)
        tile = bs.Tile(t.log2_items, t.log2_lanes, t.log2_warps, 0, 2, 0)
        for dist in workloads.DISTRIBUTIONS:
            data = workloads.make_packed(dtype, n, arrays, dist, seed=11, extremes=True)
            got = sort_with(dtype, tile, data, n, arrays, False)
            assert np.array_equal(got, expected(dtype, data, n, arrays)), (dtype, n, dist)
    assert timeouts() == t0


def test_tma_form_falls_back_when_rows_do_not_align():
    # 1000 records are 8000 bytes, not whole 128-byte rows: the one-shot kernel runs
    dtype, n, arrays = bs.I32_I32, 1000, 300
    tile = bs.Tile(5, 5, 0, 0, 2, 0)
    data = workloads.make_packed(dtype, n, arrays, "distinct16", seed=3, extremes=True)
    assert np.array_equal(sort_with(dtype, tile, data, n, arrays, False), expected(dtype, data, n, arrays))
    # an unaligned buffer start also falls back
    import torch
    d = to_device(np.concatenate([np.zeros(1, bs.NP_DTYPES[dtype]), data]))
    out = empty_device(d.numel())
    bs.sort_packed(dtype, d.data_ptr() + 8, out.data_ptr() + 8, n, arrays, 0, tile, stream_handle())
    torch.cuda.synchronize()
    got = from_device(out[8:8 + data.nbytes], bs.NP_DTYPES[dtype])
    assert np.array_equal(got, expected(dtype, data, n, arrays))


def test_tma_form_alternating_lengths_of_one_tile():
    # one kernel serves every length its tile covers; shared-memory needs differ
    # by length, so launches alternate long, short, long
    t0 = timeouts()
    dtype, tile = bs.I32_I32, bs.Tile(4, 5, 0, 0, 2, 0)     # W = 512 records
    for n in (512, 16, 512, 256, 512):
        data = workloads.make_packed(dtype, n, 700, "distinct16", seed=n, extremes=True)
        assert np.array_equal(sort_with(dtype, tile, data, n, 700, False), expected(dtype, data, n, 700)), n
    assert timeouts() == t0


def test_tma_wait_runs_out_without_a_fault():
    """Failure detection: a load that never completes (the expected byte count
    is raised above what the copy delivers) ends the bounded wait; the CTA
    counts itself, returns, and the context stays usable."""
    import torch
    stall = bs.declare("b200s_test_stall_tma_loads", ctypes.c_int, [ctypes.c_int32])
    dtype, n, arrays = bs.I32_I32, 256, 8            # one or two chunks, one CTA each
    tile = bs.Tile(4, 4, 0, 0, 2, 0)
    data = workloads.make_packed(dtype, n, arrays, "uniform", seed=5)
    before = timeouts()
    d_in = to_device(data)
    d_out = empty_device(d_in.numel())
    d_out.fill_(0)
    torch.cuda.synchronize()
    assert stall(1) == 0
    try:
        bs.sort_packed(dtype, d_in.data_ptr(), d_out.data_ptr(), n, arrays, 0, tile, stream_handle())
        torch.cuda.synchronize()
    finally:
        assert stall(0) == 0
    assert 1 <= timeouts() - before <= 2               # every CTA that gave up counted itself
    assert not from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype])["key"].any()   # chunk left unwritten
    # the device keeps working
    assert np.array_equal(sort_with(dtype, tile, data, n, arrays, False), expected(dtype, data, n, arrays))
