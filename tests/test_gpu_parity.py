"""GPU parity: the CUDA kernels, called through the C ABI, against the CPU oracle.

Bar: bit-exact.  int32/uint64 keys equal a per-array std::sort; records in
the default mode equal the reference's comparator network record for record
(tie order included); records in the stable mode equal std::stable_sort.
"""
import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device

pytestmark = pytest.mark.gpu

ALL = (bs.I32, bs.I32_I32, bs.U64, bs.U64_I32)
EDGE_N = [1, 2, 3, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 255, 256, 257,
          511, 512, 513, 1000, 1023, 1024, 1025, 2047, 2048, 2049, 4095, 4096, 4097, 8191, 8192]


def expected(dtype, flags, data, n, arrays):
    if dtype in (bs.I32, bs.U64):
        return orc.sort_packed(dtype, data, n, arrays, orc.MODE_STD, threads=8)
    mode = orc.MODE_STABLE if flags & bs.STABLE else orc.MODE_NETWORK
    return orc.sort_packed(dtype, data, n, arrays, mode, threads=8)


def gpu_sort(dtype, data, n, arrays, flags=0, tile=None, inplace=False):
    import torch
    d_in = to_device(data)
    d_out = d_in if inplace else empty_device(d_in.numel())
    bs.sort_packed(dtype, d_in.data_ptr(), d_out.data_ptr(), n, arrays, flags, tile, stream_handle())
    torch.cuda.synchronize()
    return from_device(d_out[:data.nbytes], bs.NP_DTYPES[dtype])


def check(dtype, flags, data, n, arrays, got):
    exp = expected(dtype, flags, data, n, arrays)
    assert got.shape == exp.shape
    if not np.array_equal(got, exp):
        bad = np.nonzero(got != exp)[0]
        raise AssertionError("dtype %d flags %d n %d: %d mismatches, first at %d (array %d): got %r want %r"
                             % (dtype, flags, n, len(bad), bad[0], bad[0] // n, got[bad[0]], exp[bad[0]]))
    if dtype in (bs.I32_I32, bs.U64_I32):
        if dtype == bs.I32_I32:
            off = np.arange(arrays + 1, dtype=np.int64) * n
            std = orc.sort_packed(dtype, data, n, arrays, orc.MODE_STD, threads=8)
            assert orc.validate_records(data, got, std, off) == 0


def lengths_for(dtype, flags):
    top = bs.max_length(dtype, flags)
    return [n for n in EDGE_N if n <= top] + ([top] if top not in EDGE_N else [])


@pytest.mark.parametrize("dtype", ALL)
@pytest.mark.parametrize("flags", [0, bs.STABLE])
def test_edge_lengths_uniform_with_extremes(dtype, flags):
    for n in lengths_for(dtype, flags):
        arrays = 5 if n > 2048 else 9
        data = workloads.make_packed(dtype, n, arrays, "uniform", seed=n, extremes=True)
        check(dtype, flags, data, n, arrays, gpu_sort(dtype, data, n, arrays, flags))


@pytest.mark.parametrize("dtype", ALL)
@pytest.mark.parametrize("dist", workloads.DISTRIBUTIONS)
def test_distributions(dtype, dist):
    for n in (32, 129, 256, 1000, 2048, 4096):
        for flags in (0, bs.STABLE):
            arrays = 7
            data = workloads.make_packed(dtype, n, arrays, dist, seed=3 * n + 1, extremes=True)
            check(dtype, flags, data, n, arrays, gpu_sort(dtype, data, n, arrays, flags))


@pytest.mark.parametrize("dtype", ALL)
def test_every_compiled_tile_gives_the_same_output(dtype):
    for flags in (0, bs.STABLE):
        for base in bs.tiles(dtype, flags):
            w = 1 << sum(base.as_tuple())
            for tile in (base, base.with_persistent()):
                for n in sorted({max(1, w // 2 + 1), w}):
                    arrays = 300 if w <= 256 else 4
                    data = workloads.make_packed(dtype, n, arrays, "distinct16", seed=w + n, extremes=True)
                    got = gpu_sort(dtype, data, n, arrays, flags, tile=tile)
                    check(dtype, flags, data, n, arrays, got)


@pytest.mark.parametrize("dtype", ALL)
def test_in_place(dtype):
    for n in (5, 33, 1024, 3000):
        data = workloads.make_packed(dtype, n, 6, "swap8", seed=n, extremes=True)
        check(dtype, 0, data, n, 6, gpu_sort(dtype, data, n, 6, 0, inplace=True))


def test_reference_known_answer_inputs():
    # The reference's own inputs (bench.cu:159-192, incl. EXTREMES and the
    # PERTURBED distributions) at the edge of its size sweep.
    for dist in orc.REF_DISTRIBUTIONS:
        if dist == "NORMAL":
            continue
        for n in (1, 31, 32, 33, 1023, 1024, 1025, 2048, 4096):
            arrays = 3
            for dtype, code in ((bs.I32, 0), (bs.I32_I32, 1)):
                data = orc.ref_initialize(code, n, arrays, dist, bs.NP_DTYPES[dtype])
                check(dtype, 0, data, n, arrays, gpu_sort(dtype, data, n, arrays))


def test_headline_batch_4096_by_1024_int32():
    n, arrays = 1024, 4096
    data = workloads.make_packed(bs.I32, n, arrays, "uniform", seed=2024)
    want = np.sort(data.reshape(arrays, n), axis=1)
    got = gpu_sort(bs.I32, data, n, arrays)
    assert np.array_equal(got.reshape(arrays, n), want)
    # every tile that covers n, in both launch forms (the persistent form walks
    # several arrays per group here)
    for base in bs.tiles(bs.I32):
        if (1 << sum(base.as_tuple())) < n:
            continue
        for tile in (base, base.with_persistent()):
            got = gpu_sort(bs.I32, data, n, arrays, tile=tile)
            assert np.array_equal(got.reshape(arrays, n), want), repr(tile)


def test_persistent_form_over_many_arrays_per_group():
    for dtype, n, arrays in ((bs.I32_I32, 2048, 3000), (bs.I32_I32, 100, 200000), (bs.U64_I32, 4096, 700)):
        data = workloads.make_packed(dtype, n, arrays, "distinct16", seed=arrays, extremes=True)
        tile = bs.default_tile(dtype, n).with_persistent()
        check(dtype, 0, data, n, arrays, gpu_sort(dtype, data, n, arrays, tile=tile))


@pytest.mark.parametrize("n", [32, 129, 256, 1000, 2048, 4096])
def test_record_batches_of_4m_elements_all_distributions(n):
    arrays = 4194304 // n
    for dist in workloads.DISTRIBUTIONS:
        data = workloads.make_packed(bs.I32_I32, n, arrays, dist, seed=n, extremes=True)
        got = gpu_sort(bs.I32_I32, data, n, arrays)
        check(bs.I32_I32, 0, data, n, arrays, got)


def test_large_arrays_and_multiwarp_tiles():
    for dtype in ALL:
        top = bs.max_length(dtype, 0)
        for n in (top - 1, top):
            data = workloads.make_packed(dtype, n, 3, "uniform", seed=n, extremes=True)
            check(dtype, 0, data, n, 3, gpu_sort(dtype, data, n, 3))


@pytest.mark.parametrize("dtype", [bs.I32_I32, bs.U64_I32, bs.U64])
@pytest.mark.parametrize("flags", [0, bs.STABLE])
def test_whole_warps_of_padding_are_skipped_exactly(dtype, flags):
    """Lengths whose tile has whole warps (and, for clusters, whole CTAs) of
    padding: those warps run the copy of the network that only publishes and
    synchronises.  Ties everywhere (16 distinct keys), so any moved element
    would change the output."""
    for n in (1100, 1500, 2049, 3000, 4097, 5000, 8193, 9000, 16385, 20000, 33000, 40000):
        if n > bs.max_length(dtype, flags):
            continue
        data = workloads.make_packed(dtype, n, 5, "distinct16", seed=n + 17, extremes=True)
        check(dtype, flags, data, n, 5, gpu_sort(dtype, data, n, 5, flags))


@pytest.mark.parametrize("dtype", ALL)
@pytest.mark.parametrize("flags", [0, bs.STABLE])
def test_cluster_lengths(dtype, flags):
    # arrays spanning 2..8 CTAs of a thread-block cluster
    top = bs.max_length(dtype, flags)
    assert top >= 65536
    for n in (8193, 16384, 16385, 32768, 40000, 65536, top):
        if n > top:
            continue
        data = workloads.make_packed(dtype, n, 3, "distinct16", seed=n, extremes=True)
        check(dtype, flags, data, n, 3, gpu_sort(dtype, data, n, 3, flags))


@pytest.mark.parametrize("dtype", [bs.I32_I32, bs.U64_I32])
@pytest.mark.parametrize("dist", ["uniform", "distinct16", "swap8"])
def test_cluster_batch_256_by_65536(dtype, dist):
    n, arrays = 65536, 256
    data = workloads.make_packed(dtype, n, arrays, dist, seed=65536, extremes=True)
    check(dtype, 0, data, n, arrays, gpu_sort(dtype, data, n, arrays))


def test_host_session_matches_device_path():
    import torch
    with bs.Session(0) as s:
        for dtype in ALL:
            for n, arrays in ((1, 10), (1000, 2000), (4096, 300), (129, 40000)):
                data = workloads.make_packed(dtype, n, arrays, "uniform", seed=n, extremes=True)
                pinned = torch.from_numpy(data.view(np.uint8).copy()).pin_memory()
                out = torch.empty_like(pinned).pin_memory()
                s.sort_host(dtype, pinned.data_ptr(), out.data_ptr(), n, arrays)
                got = out.numpy().view(bs.NP_DTYPES[dtype])
                check(dtype, 0, data, n, arrays, got)
                # pageable numpy buffers work too
                h_out = np.empty_like(data)
                s.sort_host(dtype, data.ctypes.data, h_out.ctypes.data, n, arrays)
                assert np.array_equal(h_out, got)


def test_host_session_ring_wraps_over_many_chunks():
    """A 327 MB batch is cut into 64 MB chunks: more chunks than device slots,
    so copy-ins wait for earlier copy-outs of the same slot."""
    import torch
    n, arrays = 4096, 20000
    data = workloads.make_packed(bs.I32, n, arrays, "uniform", seed=20000, extremes=True)
    pinned = torch.from_numpy(data.view(np.uint8).copy()).pin_memory()
    out = torch.empty_like(pinned).pin_memory()
    with bs.Session(0) as s:
        s.sort_host(bs.I32, pinned.data_ptr(), out.data_ptr(), n, arrays)
        got = out.numpy().view(bs.NP_DTYPES[bs.I32])
        assert np.array_equal(got, gpu_sort(bs.I32, data, n, arrays))
        assert np.array_equal(got.reshape(arrays, n), np.sort(data.reshape(arrays, n), axis=1))
        # the same session again with a smaller batch (slots already large enough)
        s.sort_host(bs.I32, pinned.data_ptr(), out.data_ptr(), n, 100)
        assert np.array_equal(out.numpy().view(bs.NP_DTYPES[bs.I32])[:100 * n].reshape(100, n),
                              np.sort(data[:100 * n].reshape(100, n), axis=1))
