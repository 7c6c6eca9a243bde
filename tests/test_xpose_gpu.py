"""GPU parity of launch form 3 (the transposed network, csrc/xpose.cuh)
against the oracle, through the C ABI.

Form 3 keeps every comparator layer in registers and re-lays each array out
through shared memory between register windows; keys are read striped
(coalesced), records staged through shared memory.  Bar: bit-exact -- keys
against a per-array std::sort, IntAndData records against the reference's
comparator network record for record (tie order included) -- for every
tile of every element type that has a form-3 kernel, every length the tile
covers (whole tiles, ragged tails, the sizes around each window boundary),
batches whose array count is not a multiple of the arrays per warp, in
place, misaligned buffers (which fall back to form 0), and every
distribution with the extreme keys injected.
"""
import numpy as np
import pytest

import b200sort as bs
import workloads
from test_gpu_parity import check, gpu_sort

pytestmark = pytest.mark.gpu


FORM3_TYPES = [(bs.I32, 0), (bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.U64, 0)]


def xpose_tiles(dtype, flags=0):
    out = []
    for base in bs.tiles(dtype, flags):
        if base.log2_ctas == 0 and bs.tile_info(dtype, 1 << sum(base.as_tuple()), flags, base).xpose_form:
            out.append(base.with_form(3))
    return out


def test_int32_has_form3_tiles_and_the_headline_uses_one():
    tiles = xpose_tiles(bs.I32)
    assert {1 << sum(t.as_tuple()) for t in tiles} >= {256, 512, 1024}
    assert bs.default_tile(bs.I32, 1024).persistent == 3


@pytest.mark.parametrize("dtype,flags", FORM3_TYPES)
@pytest.mark.parametrize("dist", workloads.DISTRIBUTIONS)
def test_form3_every_length_of_every_tile(dtype, flags, dist):
    tiles = xpose_tiles(dtype, flags)
    assert tiles
    for tile in tiles:
        w = 1 << sum(tile.as_tuple())
        lengths = sorted({n for n in (1, 2, 31, 32, 33, w // 32 + 1, w // 4 - 1, w // 2, w // 2 + 1, w - 33, w - 1, w)
                          if 1 <= n <= w})
        for n in lengths:
            for arrays in (1, 5, 37):
                data = workloads.make_packed(dtype, n, arrays, dist, seed=n * 7 + arrays, extremes=True)
                check(dtype, flags, data, n, arrays, gpu_sort(dtype, data, n, arrays, flags, tile))


@pytest.mark.parametrize("dtype,flags", FORM3_TYPES)
def test_form3_in_place_and_large_batches(dtype, flags):
    for tile in xpose_tiles(dtype, flags):
        w = 1 << sum(tile.as_tuple())
        for n, arrays in ((w, 20001), (w - 5, 9999)):
            data = workloads.make_packed(dtype, n, arrays, "distinct16", seed=arrays, extremes=True)
            check(dtype, flags, data, n, arrays, gpu_sort(dtype, data, n, arrays, flags, tile, inplace=True))


def test_form3_misaligned_record_buffers_fall_back():
    import torch
    from gpu_util import from_device, stream_handle, to_device
    n, arrays = 1000, 64
    tile = bs.default_tile(bs.I32_I32, n).with_form(3)
    data = workloads.make_packed(bs.I32_I32, n, arrays, "distinct16", seed=8, extremes=True)
    raw = to_device(data)
    d_in = torch.zeros(raw.numel() + 4, dtype=torch.uint8, device="cuda")
    d_in[4:].copy_(raw)                       # records 4 bytes off their 8-byte alignment
    d_out = torch.zeros_like(d_in)
    bs.sort_packed(bs.I32_I32, d_in.data_ptr() + 4, d_out.data_ptr() + 4, n, arrays, 0, tile, stream_handle())
    torch.cuda.synchronize()
    check(bs.I32_I32, 0, data, n, arrays, from_device(d_out[4:], bs.NP_DTYPES[bs.I32_I32]))


def test_form3_headline_batch_default_path():
    n, arrays = 1024, 4096
    data = workloads.make_packed(bs.I32, n, arrays, "uniform", seed=77)
    got = gpu_sort(bs.I32, data, n, arrays)
    assert np.array_equal(got.reshape(arrays, n), np.sort(data.reshape(arrays, n), axis=1))


def test_form3_request_on_a_tile_without_it_falls_back():
    # uint64-key records have no single-warp form-3 kernel: the request runs
    # form 0, same output
    n, arrays = 300, 50
    data = workloads.make_packed(bs.U64_I32, n, arrays, "distinct16", seed=3, extremes=True)
    tile = bs.default_tile(bs.U64_I32, n).with_form(3)
    assert not bs.tile_info(bs.U64_I32, n, 0, tile).xpose_form
    check(bs.U64_I32, 0, data, n, arrays, gpu_sort(bs.U64_I32, data, n, arrays, 0, tile))
