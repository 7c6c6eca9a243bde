"""GPU parity of the ragged (CSR) path: the persistent bucketed launch (graph
replay and direct), and the plain per-length launches, against the oracle."""
import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device

pytestmark = pytest.mark.gpu

ALL = (bs.I32, bs.I32_I32, bs.U64, bs.U64_I32)


def expected(dtype, flags, data, off):
    if dtype in (bs.I32, bs.U64):
        return orc.sort_ragged(dtype, data, off, orc.MODE_STD, threads=16)
    mode = orc.MODE_STABLE if flags & bs.STABLE else orc.MODE_NETWORK
    return orc.sort_ragged(dtype, data, off, mode, threads=16)


def run(dtype, flags, data, off, form="graph", plan=None, reps=1):
    import torch
    d_in = to_device(data)
    d_out = empty_device(d_in.numel())
    d_off = torch.from_numpy(off.astype(np.int32)).cuda()
    own = plan is None
    plan = plan or bs.Plan(dtype, len(off) - 1, flags | (bs.PLAN_NO_GRAPH if form == "direct" else 0))
    st = stream_handle()
    if form == "plain":
        plan.prepare_plain(off.astype(np.int32))
    for _ in range(reps):
        if form == "plain":
            plan.sort_plain(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), st)
        else:
            plan.sort(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), len(off) - 1, st)
    torch.cuda.synchronize()
    too_long = plan.too_long(st) if form != "plain" else 0
    if own:
        plan.close()
    return from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype]), too_long


def check(dtype, flags, data, off, got):
    exp = expected(dtype, flags, data, off)
    if not np.array_equal(got, exp):
        bad = np.nonzero(got != exp)[0]
        a = np.searchsorted(off, bad[0], side="right") - 1
        raise AssertionError("dtype %d flags %d: %d mismatches, first at %d (array %d, n %d)"
                             % (dtype, flags, len(bad), bad[0], a, off[a + 1] - off[a]))
    if dtype == bs.I32_I32:
        std = orc.sort_ragged(dtype, data, off, orc.MODE_STD, threads=16)
        assert orc.validate_records(data, got, std, off) == 0


@pytest.mark.parametrize("dtype", ALL)
@pytest.mark.parametrize("flags", [0, bs.STABLE])
@pytest.mark.parametrize("form", ["graph", "direct", "plain"])
def test_ragged_forms_match_oracle(dtype, flags, form):
    top = bs.ragged_max_length(dtype, flags)
    lengths = workloads.ragged_lengths(1500, max_len=top, seed=dtype * 10 + flags)
    lengths[::97] = 0                      # empty arrays
    lengths[5] = top                       # the largest bucket, full
    lengths[6] = 1
    data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=7, extremes=True)
    got, too_long = run(dtype, flags, data, off, form)
    assert too_long == 0
    check(dtype, flags, data, off, got)


@pytest.mark.parametrize("dtype", [bs.I32, bs.I32_I32])
def test_every_length_up_to_600(dtype):
    lengths = np.arange(0, 601)
    data, off = workloads.make_ragged(dtype, lengths, "uniform", seed=3, extremes=True)
    for form in ("graph", "plain"):
        got, _ = run(dtype, 0, data, off, form)
        check(dtype, 0, data, off, got)


def test_graph_replay_and_recapture():
    import torch
    dtype = bs.I32_I32
    lengths = workloads.ragged_lengths(800, max_len=4096, seed=11)
    data, off = workloads.make_ragged(dtype, lengths, "swap8", seed=12, extremes=True)
    exp = expected(dtype, 0, data, off)
    with bs.Plan(dtype, 2000) as plan:
        st = stream_handle()
        d_off = torch.from_numpy(off.astype(np.int32)).cuda()
        a_in, b_in = to_device(data), to_device(data)
        a_out, b_out = empty_device(a_in.numel()), empty_device(a_in.numel())
        for _ in range(3):                  # replays of one graph
            plan.sort(a_in.data_ptr(), a_out.data_ptr(), d_off.data_ptr(), len(lengths), st)
        plan.sort(b_in.data_ptr(), b_out.data_ptr(), d_off.data_ptr(), len(lengths), st)   # re-capture
        plan.sort(a_in.data_ptr(), a_in.data_ptr(), d_off.data_ptr(), len(lengths), st)    # in place
        torch.cuda.synchronize()
        for t in (a_out, b_out, a_in):
            assert np.array_equal(from_device(t[:data.nbytes], bs.NP_DTYPES[dtype]), exp)
        # fewer arrays than the plan holds: a prefix of the batch
        k = 300
        c_out = empty_device(a_in.numel())
        plan.sort(b_in.data_ptr(), c_out.data_ptr(), d_off.data_ptr(), k, st)
        torch.cuda.synchronize()
        got = from_device(c_out[:data.nbytes], bs.NP_DTYPES[dtype])
        assert np.array_equal(got[:off[k]], exp[:off[k]])


def test_too_long_arrays_are_reported_and_left_alone():
    dtype = bs.I32
    top = bs.ragged_max_length(dtype)
    lengths = np.array([10, top + 1, 20, 3 * top, 5], dtype=np.int64)
    data, off = workloads.make_ragged(dtype, lengths, "uniform", seed=1)
    got, too_long = run(dtype, 0, data, off, "graph")
    assert too_long == 2
    for a in (0, 2, 4):
        lo, hi = off[a], off[a + 1]
        assert np.array_equal(got[lo:hi], np.sort(data[lo:hi]))


def test_full_ragged_batch_200000_arrays():
    dtype = bs.I32_I32
    lengths = workloads.ragged_lengths(200000, max_len=8192, seed=1234)
    data, off = workloads.make_ragged(dtype, lengths, "uniform", seed=1234)
    got, too_long = run(dtype, 0, data, off, "graph", reps=2)
    assert too_long == 0
    check(dtype, 0, data, off, got)


def _route(dtype, flags, rows):
    """Load ragged table rows (log2 W, family) for dtype/flags; family 2 gives
    the bucket its own launch of the tabled tile."""
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        for L, fam in rows:
            f.write("r,%d,%d,%d,%d\n" % (dtype, flags, L, fam))
    try:
        bs.load_tile_table(f.name)
    finally:
        import os
        os.unlink(f.name)


@pytest.mark.parametrize("dtype,flags", [(bs.I32, 0), (bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.U64, 0),
                                         (bs.U64_I32, 0)])
def test_buckets_with_their_own_launch_match_the_oracle(dtype, flags):
    # every persistent-range bucket dedicated, then every other one, then none:
    # the same output, record for record, in the graph and the direct form
    top = bs.ragged_max_length(dtype, flags)
    lengths = workloads.ragged_lengths(4000, max_len=min(top, 12000), seed=31)
    lengths[::29] = 0
    data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=31, extremes=True)
    exp = expected(dtype, flags, data, off)
    Ls = list(range(3, 15))
    try:
        for routing in ([(L, 2) for L in Ls], [(L, 2 if L % 2 else 0) for L in Ls]):
            _route(dtype, flags, routing)
            for form in ("graph", "direct"):
                got, too_long = run(dtype, flags, data, off, form, reps=2)
                assert too_long == 0
                assert np.array_equal(got, exp), (routing[:2], form)
            # the allocation-free path follows the same routing
            import ctypes
            import torch
            fn = bs.declare("b200s_sort_ragged_noalloc", ctypes.c_int,
                            [ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_int64, ctypes.c_void_p])
            d_in = to_device(data)
            d_out = empty_device(d_in.numel())
            d_off = torch.from_numpy(off.astype(np.int32)).cuda()
            assert fn(dtype, flags, d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), len(off) - 1,
                      stream_handle()) == 0
            torch.cuda.synchronize()
            assert np.array_equal(from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype]), exp)
    finally:
        _route(dtype, flags, [(L, 0) for L in Ls])
        import os
        table = os.path.join(os.path.dirname(bs.LIB_PATH), "tune", "b200_table.csv")
        bs.load_tile_table(table)   # back to the shipped table


@pytest.mark.parametrize("dtype,flags", [(bs.I32, 0), (bs.I32_I32, 0), (bs.U64_I32, bs.STABLE)])
def test_hinted_sort_launches_only_the_classes_present(dtype, flags):
    # a direct plan told the host offsets skips the empty classes: batches with
    # only short arrays, only long ones, only cluster-range ones, a mix, and
    # only empty arrays, under the shipped routing and with every other
    # persistent-range class on a launch of its own
    import os
    import torch
    top = bs.ragged_max_length(dtype, flags)
    rng = np.random.default_rng(77)
    cases = [rng.integers(1, 33, 300), rng.integers(2049, 8193, 40), rng.integers(16385, top + 1, 6),
             np.concatenate([rng.integers(1, 17, 50), rng.integers(4097, 8193, 8), rng.integers(16385, top + 1, 3)]),
             np.array([0] * 19 + [5]), np.array([1000])]
    Ls = list(range(3, 15))
    plan = bs.Plan(dtype, 400, flags | bs.PLAN_NO_GRAPH)
    st = stream_handle()
    try:
        for routing in (None, [(L, 2 if L % 2 else 0) for L in Ls]):
            if routing:
                plan.close()
                _route(dtype, flags, routing)
                plan = bs.Plan(dtype, 400, flags | bs.PLAN_NO_GRAPH)
            for i, lengths in enumerate(cases):
                lengths = rng.permutation(lengths.astype(np.int64))
                data, off = workloads.make_ragged(dtype, lengths, "uniform", seed=i, extremes=True)
                exp = expected(dtype, flags, data, off)
                d_in = to_device(data)
                d_out = to_device(np.zeros_like(data))
                d_off = torch.from_numpy(off.astype(np.int32)).cuda()
                plan.sort_hinted(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), off.astype(np.int32), st)
                torch.cuda.synchronize()
                assert plan.too_long(st) == 0
                got = from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype])
                assert np.array_equal(got, exp), (routing is not None, i)
    finally:
        plan.close()
        _route(dtype, flags, [(L, 0) for L in Ls])
        bs.load_tile_table(os.path.join(os.path.dirname(bs.LIB_PATH), "tune", "b200_table.csv"))


@pytest.mark.parametrize("dtype,flags", [(bs.I32, 0), (bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.U64_I32, 0)])
def test_launch_of_its_own_in_every_named_tile_and_form(dtype, flags):
    # ragged rows that name the tile and form of a class's own launch: every
    # single-CTA tile of W = 512 .. 4096 in forms 0 and 3 (where compiled)
    # gives the oracle's output, graph and direct
    import os
    lengths = workloads.ragged_lengths(3000, max_len=4096, seed=41)
    data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=41, extremes=True)
    exp = expected(dtype, flags, data, off)
    cands = []
    for t in bs.tiles(dtype, flags):
        L = sum(t.as_tuple())
        if t.log2_ctas == 0 and 9 <= L <= 12:
            info = bs.tile_info(dtype, 1 << L, flags, t)
            for form in ([0] if info.arrays_per_cta else []) + ([3] if info.xpose_form else []):
                cands.append((L, t, form))
    assert cands
    try:
        for L, t, form in cands:
            _own = "r,%d,%d,%d,2,%d,%d,%d,%d" % (dtype, flags, L, t.log2_items, t.log2_lanes, t.log2_warps, form)
            import tempfile
            with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
                f.write(_own + "\n")
            bs.load_tile_table(f.name)
            os.unlink(f.name)
            for mode in ("graph", "direct"):
                got, too_long = run(dtype, flags, data, off, mode)
                assert too_long == 0
                assert np.array_equal(got, exp), (_own, mode)
    finally:
        bs.load_tile_table(os.path.join(os.path.dirname(bs.LIB_PATH), "tune", "b200_table.csv"))
