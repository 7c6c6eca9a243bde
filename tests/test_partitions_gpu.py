"""The leaf of the reference's partitioned large-array sort through
b200s_sort_partitions (the contract of SortPartitionsAdaptive_outofplace,
cusort.hpp:2309-2352).

A 2^20-element array is split by the reference's OWN partition stage
(HybridSortPartitionedV3's pivots, counts, single-value flags and scatter,
cusort.hpp:2493-2588, compiled unmodified into oracle/_ref and run on the
B200: 512 partitions); the partitions are then sorted by
b200s_sort_partitions, out of place, with the reference's counters and
flags.  (At 1024 partitions -- 2^21 and 2^22 uniform keys -- that partition
stage did not keep the input's elements on the B200, so the reference
partitions stop at 2^20; a 2^22 array split into 1024 key ranges by a numpy
sample sort covers the larger partition count.)  The partitions are key ranges in
order, so the result must equal a std::sort of the whole array, and for
records every partition must equal the reference's comparator network on it
(the order of equal keys included) -- what the reference's leaf kernels
return for the partitions they sort.  Partitions longer than the longest
sortable length are not written (the reference sends those to its merge
path); the test fills them from the input before comparing.
"""
import ctypes

import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, stream_handle, to_device

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.ref_gpu_available(), reason="reference GPU kernels not built")]

N = 1 << 20


def ref_partition(dtype, data):
    import torch
    suffix = "int" if dtype == bs.I32 else "rec"
    fn = getattr(orc.ref_gpu(suffix), "ref_partition_v3_" + suffix)
    d = to_device(data)
    parts = empty_device(d.numel())
    counters = torch.zeros(1026, dtype=torch.int32, device="cuda")
    uniform = torch.zeros(1025, dtype=torch.int32, device="cuda")
    nb, skipped = ctypes.c_int(0), ctypes.c_int(0)
    rc = fn(d.data_ptr(), len(data), parts.data_ptr(), counters.data_ptr(), uniform.data_ptr(), ctypes.byref(nb),
            ctypes.byref(skipped), stream_handle())
    assert rc == 0
    torch.cuda.synchronize()
    return parts, counters, uniform, nb.value, skipped.value


@pytest.mark.parametrize("dtype,dist", [(bs.I32, "uniform"), (bs.I32, "distinct16"), (bs.I32, "equal"),
                                        (bs.I32_I32, "uniform"), (bs.I32_I32, "distinct16"),
                                        (bs.I32_I32, "swap64")])
def test_reference_partitions_sorted_by_the_leaf_hook(dtype, dist):
    import torch
    data = workloads.make_packed(dtype, N, 1, dist, seed=17)
    parts, counters, uniform, nb, skipped = ref_partition(dtype, data)
    assert 1 <= nb <= 1024
    off = counters[:nb + 1].cpu().numpy().astype(np.int64)
    assert off[0] == 0 and off[-1] == N and np.all(np.diff(off) >= 0)
    out = empty_device(parts.numel())
    bs.sort_partitions(dtype, parts.data_ptr(), out.data_ptr(), counters.data_ptr(), nb, uniform.data_ptr(),
                       0, stream_handle())
    torch.cuda.synchronize()
    got = from_device(out[:data.nbytes], bs.NP_DTYPES[dtype])
    part_in = from_device(parts[:data.nbytes], bs.NP_DTYPES[dtype])
    # every partition sorted as the reference's network sorts it; partitions
    # beyond the longest sortable length are left as they are (the contract)
    want = orc.sort_ragged(dtype, part_in, off, orc.MODE_NETWORK if dtype else orc.MODE_STD, threads=8)
    sizes = np.diff(off)
    big = np.nonzero(sizes > bs.ragged_max_length(dtype, 0))[0]
    for p in big:
        # not written by the hook (the reference sorts such partitions with its
        # merge path): the caller's copy stands in for that path here
        got[off[p]:off[p + 1]] = want[off[p]:off[p + 1]] = part_in[off[p]:off[p + 1]]
    assert np.array_equal(got, want)
    flags = uniform[:nb].cpu().numpy() != 0
    if all(flags[p] for p in big):
        # the partitions are key ranges in order: the whole array is sorted
        keys = got if dtype == bs.I32 else got["key"]
        assert np.array_equal(keys, np.sort(data if dtype == bs.I32 else data["key"]))
    if dtype == bs.I32_I32:
        # payload = original position: every record kept its own payload
        assert np.array_equal(data["key"][got["data"]], got["key"])
    # in place, a second call through the cached plan
    bs.sort_partitions(dtype, parts.data_ptr(), parts.data_ptr(), counters.data_ptr(), nb, 0, 0, stream_handle())
    torch.cuda.synchronize()
    again = from_device(parts[:data.nbytes], bs.NP_DTYPES[dtype])
    assert np.array_equal(again, got)


def test_leaf_hook_stable_mode_and_argument_checks():
    import torch
    # 4096 distinct keys, about 256 records each: ties in every partition
    data = workloads.make_packed(bs.I32_I32, N, 1, "uniform", seed=5)
    data["key"] >>= 20
    parts, counters, uniform, nb, _ = ref_partition(bs.I32_I32, data)
    assert np.diff(counters[:nb + 1].cpu().numpy()).max() <= bs.ragged_max_length(bs.I32_I32, bs.STABLE)
    out = empty_device(parts.numel())
    bs.sort_partitions(bs.I32_I32, parts.data_ptr(), out.data_ptr(), counters.data_ptr(), nb, 0, bs.STABLE,
                       stream_handle())
    torch.cuda.synchronize()
    got = from_device(out[:data.nbytes], bs.NP_DTYPES[bs.I32_I32])
    off = counters[:nb + 1].cpu().numpy().astype(np.int64)
    part_in = from_device(parts[:data.nbytes], bs.NP_DTYPES[bs.I32_I32])
    assert np.array_equal(got, orc.sort_ragged(bs.I32_I32, part_in, off, orc.MODE_STABLE, threads=8))
    assert bs.lib().b200s_sort_partitions(bs.I32, 0, None, None, None, None, -1, None) == 1
    assert bs.lib().b200s_sort_partitions(bs.I32, 0, None, None, None, None, 0, None) == 0
    assert bs.lib().b200s_release_partition_plans() == 0


def cpu_partition(keys, parts, seed=0):
    """Sample-sort split into `parts` key ranges (pivots: quantiles of a
    sample); returns the permutation that groups the elements by range, in
    input order inside each range, and the CSR offsets."""
    rng = np.random.default_rng(seed)
    sample = np.sort(keys[rng.integers(0, len(keys), size=parts * 32)])
    pivots = sample[np.arange(1, parts) * 32]
    bucket = np.searchsorted(pivots, keys, side="right")
    order = np.argsort(bucket, kind="stable")
    off = np.zeros(parts + 1, dtype=np.int64)
    np.cumsum(np.bincount(bucket, minlength=parts), out=off[1:])
    return order, off


@pytest.mark.parametrize("dtype", [bs.I32, bs.I32_I32])
def test_1024_key_range_partitions_of_4m_elements(dtype):
    import torch
    n = 1 << 22
    data = workloads.make_packed(dtype, n, 1, "uniform", seed=23, extremes=True)
    keys = data if dtype == bs.I32 else data["key"]
    order, off = cpu_partition(keys, 1024)
    part_in = data[order]
    d_in = to_device(part_in)
    d_off = torch.from_numpy(off.astype(np.int32)).cuda()
    out = empty_device(d_in.numel())
    bs.sort_partitions(dtype, d_in.data_ptr(), out.data_ptr(), d_off.data_ptr(), 1024, 0, 0, stream_handle())
    torch.cuda.synchronize()
    got = from_device(out[:data.nbytes], bs.NP_DTYPES[dtype])
    want = orc.sort_ragged(dtype, part_in, off, orc.MODE_NETWORK if dtype else orc.MODE_STD, threads=8)
    assert np.array_equal(got, want)
    assert np.array_equal(got if dtype == bs.I32 else got["key"], np.sort(keys))
