"""B200S_SORTED_CHECK (the reference's Sorted switch, cusort_v6.hpp:103-128):
the packed path tests each array before sorting (the transposed-network form
also after every stage of span >= 16) and skips the rest once it is in
order.  A tile in order is a fixed point of the network, so the output must
be identical with and without the flag, bit for bit, on every distribution,
for every element type and launch form; arrays already in order sorted in
place must be left untouched.
"""
import numpy as np
import pytest

import b200sort as bs
import workloads
from test_gpu_parity import check, gpu_sort

pytestmark = pytest.mark.gpu

CHECK = bs.SORTED_CHECK if hasattr(bs, "SORTED_CHECK") else 2
LENGTHS = [1, 31, 32, 100, 129, 256, 1000, 1024, 2048, 4096]


@pytest.mark.parametrize("dtype,flags", [(bs.I32, 0), (bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.U64, 0),
                                         (bs.U64_I32, 0), (bs.U64_I32, bs.STABLE)])
@pytest.mark.parametrize("dist", workloads.DISTRIBUTIONS)
def test_flag_changes_no_output(dtype, flags, dist):
    for n in LENGTHS:
        if n > bs.max_length(dtype, flags):
            continue
        arrays = 7
        for extremes in (False, True):
            data = workloads.make_packed(dtype, n, arrays, dist, seed=n + 11, extremes=extremes)
            plain = gpu_sort(dtype, data, n, arrays, flags)
            checked = gpu_sort(dtype, data, n, arrays, flags | CHECK)
            assert np.array_equal(plain, checked), (dtype, flags, dist, n, extremes)
            check(dtype, flags, data, n, arrays, checked)


@pytest.mark.parametrize("form", [0, 1, 2, 3])
def test_every_launch_form_with_the_flag(form):
    for dtype in (bs.I32, bs.I32_I32):
        for n in (256, 1024):
            tile = bs.default_tile(dtype, n).with_form(form)
            for dist in ("sorted", "equal", "swap1", "uniform"):
                data = workloads.make_packed(dtype, n, 300, dist, seed=n)
                want = gpu_sort(dtype, data, n, 300, 0, tile)
                got = gpu_sort(dtype, data, n, 300, CHECK, tile)
                assert np.array_equal(got, want), (dtype, n, form, dist)
                check(dtype, 0, data, n, 300, got)


def test_sorted_arrays_in_place_are_left_untouched():
    for dtype in (bs.I32, bs.I32_I32, bs.U64_I32):
        for n in (64, 1000, 1024, 2048):
            data = workloads.make_packed(dtype, n, 50, "sorted", seed=5)
            got = gpu_sort(dtype, data, n, 50, CHECK, inplace=True)
            assert np.array_equal(got, data)


def test_partly_sorted_batches_mix_skipped_and_sorted_arrays():
    # every other array already in order: both kinds in one warp / one launch
    for dtype in (bs.I32, bs.I32_I32):
        for n in (32, 256, 1024):
            a = workloads.make_packed(dtype, n, 64, "sorted", seed=1).reshape(64, n)
            b = workloads.make_packed(dtype, n, 64, "uniform", seed=2).reshape(64, n)
            mix = a.copy()
            mix[1::2] = b[1::2]
            data = mix.reshape(-1)
            check(dtype, 0, data, n, 64, gpu_sort(dtype, data, n, 64, CHECK))
            check(dtype, 0, data, n, 64, gpu_sort(dtype, data, n, 64, CHECK, inplace=True))
