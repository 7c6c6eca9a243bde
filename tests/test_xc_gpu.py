"""GPU parity of launch form 3 on multi-warp and cluster tiles (the transposed
network of csrc/cta_xpose.cuh) against the oracle, through the C ABI.

Every comparator layer runs in registers; the tile moves between register
windows through one padded shared-memory region per CTA, and cluster tiles
exchange across CTAs through distributed shared memory.  Bar: bit-exact --
keys against a per-array std::sort, records against the reference's
comparator network record for record (tie order included) -- for every
multi-warp and cluster tile of every element type, lengths around the
window and CTA boundaries, several arrays per launch, in place, and the
ragged plan's dedicated and cluster launches when the tile table picks
form 3 for their lengths.
"""
import os
import tempfile

import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device
from test_gpu_parity import check, gpu_sort

pytestmark = pytest.mark.gpu

ALL = [(d, f) for d in (bs.I32, bs.I32_I32, bs.U64, bs.U64_I32) for f in (0, bs.STABLE)]


def xc_tiles(dtype, flags):
    out = []
    for base in bs.tiles(dtype, flags):
        w = 1 << sum(base.as_tuple())
        if (base.log2_warps > 0 or base.log2_ctas > 0) and bs.tile_info(dtype, w, flags, base).xpose_form:
            out.append(base.with_form(3))
    return out


def width(tile):
    return 1 << sum(tile.as_tuple())


def test_every_type_has_multi_warp_and_cluster_form3_tiles():
    for dtype, flags in ALL:
        tiles = xc_tiles(dtype, flags)
        assert any(t.log2_ctas == 0 for t in tiles), (dtype, flags)
        assert any(t.log2_ctas > 0 for t in tiles) or dtype == bs.I32, (dtype, flags)


@pytest.mark.parametrize("dtype,flags", ALL)
@pytest.mark.parametrize("dist", ["uniform", "distinct16", "sorted", "organ", "swap8"])
def test_form3_multi_warp_and_cluster_tiles(dtype, flags, dist):
    for tile in xc_tiles(dtype, flags):
        w = width(tile)
        lengths = sorted({n for n in (w // 2 + 1, w // 2 + 257, w - 17, w) if n >= 1})
        for n in lengths:
            arrays = 3 if w >= 32768 else 7
            data = workloads.make_packed(dtype, n, arrays, dist, seed=n + w + arrays, extremes=True)
            check(dtype, flags, data, n, arrays, gpu_sort(dtype, data, n, arrays, flags, tile))


@pytest.mark.parametrize("dtype,flags", ALL)
def test_form3_in_place_and_batches_wider_than_the_gpu(dtype, flags):
    for tile in xc_tiles(dtype, flags):
        w = width(tile)
        arrays = max(3, (8 << 20) // (w * 8))   # about 8 M elements' worth of arrays
        arrays = min(arrays, 600)
        data = workloads.make_packed(dtype, w, arrays, "distinct16", seed=w + 1, extremes=True)
        check(dtype, flags, data, w, arrays, gpu_sort(dtype, data, w, arrays, flags, tile, inplace=True))


def _table(rows):
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        for r in rows:
            f.write(",".join(str(x) for x in r) + "\n")
    try:
        bs.load_tile_table(f.name)
    finally:
        os.unlink(f.name)


def _restore():
    bs.load_tile_table(os.path.join(os.path.dirname(bs.LIB_PATH), "tune", "b200_table.csv"))


@pytest.mark.parametrize("dtype,flags", [(bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.U64_I32, 0), (bs.U64, 0)])
def test_ragged_plan_runs_form3_for_its_classes(dtype, flags):
    # every length class with a form-3 tile (one-warp, multi-warp) on a launch
    # of its own in that form, and the cluster classes in form 3: graph,
    # direct, hinted, plain per class and the allocation-free path all equal
    # the oracle
    import ctypes
    import torch
    top = bs.ragged_max_length(dtype, flags)
    rows = []
    one_warp = [b.with_form(3) for b in bs.tiles(dtype, flags)
                if b.log2_warps == 0 and b.log2_ctas == 0 and b.log2_lanes > 0
                and bs.tile_info(dtype, 1 << sum(b.as_tuple()), flags, b).xpose_form]
    for tile in one_warp + xc_tiles(dtype, flags):
        w = width(tile)
        L = w.bit_length() - 1
        rows.append((dtype, flags, L) + tile.as_tuple()[:3] + (3, tile.log2_ctas))
        if tile.log2_ctas == 0:
            rows.append(("r", dtype, flags, L, 2))
    try:
        _table(rows)
        rng = np.random.default_rng(5)
        lengths = np.concatenate([rng.integers(1, 600, 400), rng.integers(600, 8193, 120),
                                  rng.integers(8193, top + 1, 6), np.array([0, 1, top])])
        lengths = rng.permutation(lengths)
        data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=9, extremes=True)
        if dtype in (bs.I32, bs.U64):
            exp = orc.sort_ragged(dtype, data, off, orc.MODE_STD, threads=16)
        else:
            mode = orc.MODE_STABLE if flags & bs.STABLE else orc.MODE_NETWORK
            exp = orc.sort_ragged(dtype, data, off, mode, threads=16)
        off32 = off.astype(np.int32)
        d_off = torch.from_numpy(off32).cuda()
        st = stream_handle()
        for form in ("graph", "direct", "hinted", "plain"):
            plan = bs.Plan(dtype, len(off) - 1, flags | (0 if form == "graph" else bs.PLAN_NO_GRAPH))
            d_in = to_device(data)
            d_out = empty_device(d_in.numel())
            if form == "plain":
                plan.prepare_plain(off32, by_bucket=True)
                plan.sort_plain(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), st)
            elif form == "hinted":
                plan.sort_hinted(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), off32, st)
            else:
                plan.sort(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), len(off) - 1, st)
            torch.cuda.synchronize()
            plan.close()
            got = from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype])
            assert np.array_equal(got, exp), form
        fn = bs.declare("b200s_sort_ragged_noalloc", ctypes.c_int,
                        [ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                         ctypes.c_int64, ctypes.c_void_p])
        d_in = to_device(data)
        d_out = empty_device(d_in.numel())
        assert fn(dtype, flags, d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), len(off) - 1, st) == 0
        torch.cuda.synchronize()
        assert np.array_equal(from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype]), exp)
    finally:
        _restore()
