"""GPU parity of launch form 3 (the transposed network, csrc/xpose.cuh)
against the oracle, through the C ABI.

Form 3 keeps every comparator layer in registers and re-lays each array out
through shared memory between register windows; int32 keys are read and
written striped (coalesced).  Bar: bit-exact against a per-array std::sort,
for every tile that has a form-3 kernel, every length the tile covers
(whole tiles, ragged tails, the sizes around each window boundary), batches
whose array count is not a multiple of the arrays per warp, in place, and
every distribution with the extreme keys injected.
"""
import numpy as np
import pytest

import b200sort as bs
import workloads
from test_gpu_parity import check, gpu_sort

pytestmark = pytest.mark.gpu


def xpose_tiles(dtype):
    out = []
    for base in bs.tiles(dtype):
        if base.log2_ctas == 0 and bs.tile_info(dtype, 1 << sum(base.as_tuple()), 0, base).xpose_form:
            out.append(base.with_form(3))
    return out


def test_int32_has_form3_tiles_and_the_headline_uses_one():
    tiles = xpose_tiles(bs.I32)
    assert {1 << sum(t.as_tuple()) for t in tiles} >= {256, 512, 1024}
    assert bs.default_tile(bs.I32, 1024).persistent == 3


@pytest.mark.parametrize("dist", workloads.DISTRIBUTIONS)
def test_form3_every_length_of_every_tile(dist):
    for tile in xpose_tiles(bs.I32):
        w = 1 << sum(tile.as_tuple())
        lengths = sorted({1, 2, 31, 32, 33, w // 32 + 1, w // 4 - 1, w // 2, w // 2 + 1, w - 33, w - 1, w})
        for n in lengths:
            for arrays in (1, 5, 37):
                data = workloads.make_packed(bs.I32, n, arrays, dist, seed=n * 7 + arrays, extremes=True)
                check(bs.I32, 0, data, n, arrays, gpu_sort(bs.I32, data, n, arrays, tile=tile))


def test_form3_in_place_and_large_batches():
    for tile in xpose_tiles(bs.I32):
        w = 1 << sum(tile.as_tuple())
        for n, arrays in ((w, 20001), (w - 5, 9999)):
            data = workloads.make_packed(bs.I32, n, arrays, "uniform", seed=arrays, extremes=True)
            want = np.sort(data.reshape(arrays, n), axis=1)
            got = gpu_sort(bs.I32, data, n, arrays, tile=tile, inplace=True)
            assert np.array_equal(got.reshape(arrays, n), want), repr(tile)


def test_form3_headline_batch_default_path():
    n, arrays = 1024, 4096
    data = workloads.make_packed(bs.I32, n, arrays, "uniform", seed=77)
    got = gpu_sort(bs.I32, data, n, arrays)
    assert np.array_equal(got.reshape(arrays, n), np.sort(data.reshape(arrays, n), axis=1))


def test_form3_request_on_a_tile_without_it_falls_back():
    # records have no form-3 kernel: the request runs form 0, same output
    n, arrays = 1000, 50
    data = workloads.make_packed(bs.I32_I32, n, arrays, "distinct16", seed=3, extremes=True)
    tile = bs.default_tile(bs.I32_I32, n).with_form(3)
    check(bs.I32_I32, 0, data, n, arrays, gpu_sort(bs.I32_I32, data, n, arrays, tile=tile))
