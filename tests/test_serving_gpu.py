"""GPU tests of the serving path (b200s_server_*): every request's result is
the same sorted alone and sorted inside a mix of concurrent requests of
other sizes, and equals the oracle (bit for bit: the network's tie order for
records, std::stable_sort in the stable mode).  Also host-memory requests,
the device-memory budget and the request-level errors."""
import threading

import numpy as np
import pytest

import b200sort as bs
import cpu_oracle as orc
import workloads
from gpu_util import empty_device, from_device, to_device

pytestmark = pytest.mark.gpu


def make_requests(dtype, count, seed, max_len=65536):
    """Requests of lengths log-uniform in [16, max_len] (a few of each size
    class), keys from 16 distinct values plus the extremes: many ties."""
    max_len = min(max_len, bs.ragged_max_length(dtype))
    lengths = workloads.log_uniform_lengths(count, 16, max_len, seed=seed)
    lengths[:4] = [1, 2, 8193, max_len] if max_len >= 8193 else [1, 2, 3, max_len]
    data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=seed, extremes=True)
    return [data[off[i]:off[i + 1]].copy() for i in range(count)]


def expected_one(dtype, flags, arr):
    off = np.array([0, len(arr)], dtype=np.int64)
    if dtype in (bs.I32, bs.U64):
        mode = orc.MODE_STD
    else:
        mode = orc.MODE_STABLE if flags & bs.STABLE else orc.MODE_NETWORK
    return orc.sort_ragged(dtype, arr, off, mode)


def sort_alone(srv, dtype, reqs):
    import torch
    outs = []
    for arr in reqs:
        d_in = to_device(arr)
        d_out = empty_device(arr.nbytes)
        t = srv.submit(d_in.data_ptr(), d_out.data_ptr(), len(arr))
        assert srv.wait(t, 60_000_000) == bs.OK
        torch.cuda.synchronize()
        outs.append(from_device(d_out[:arr.nbytes], bs.NP_DTYPES[dtype]))
    return outs


def sort_in_mix(srv, dtype, reqs, threads=3):
    """All requests submitted at once from several host threads."""
    import torch
    d_in = [to_device(a) for a in reqs]
    d_out = [empty_device(a.nbytes) for a in reqs]
    torch.cuda.synchronize()
    tickets = [None] * len(reqs)

    def client(k):
        for i in range(k, len(reqs), threads):
            tickets[i] = srv.submit(d_in[i].data_ptr(), d_out[i].data_ptr(), len(reqs[i]))

    th = [threading.Thread(target=client, args=(k,)) for k in range(threads)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for t in tickets:
        assert srv.wait(t, 60_000_000) == bs.OK
    torch.cuda.synchronize()
    return [from_device(d_out[i][:reqs[i].nbytes], bs.NP_DTYPES[dtype]) for i in range(len(reqs))]


@pytest.mark.parametrize("dtype,flags", [(bs.I32_I32, 0), (bs.I32_I32, bs.STABLE), (bs.I32, 0), (bs.U64, 0),
                                         (bs.U64_I32, 0)])
def test_result_alone_equals_result_in_mix(dtype, flags):
    reqs = make_requests(dtype, 120, seed=7 + dtype)
    with bs.Server(dtype, budget_bytes=256 << 20, max_inflight=4, max_batch=64, flags=flags) as srv:
        alone = sort_alone(srv, dtype, reqs)
        mixed = sort_in_mix(srv, dtype, reqs)
        s = srv.stats()
        assert s.failed == 0 and s.completed == 2 * len(reqs)
        assert s.max_batch_requests > 1      # the mix formed multi-request batches
    for i, arr in enumerate(reqs):
        want = expected_one(dtype, flags, arr)
        assert np.array_equal(alone[i], want), "request %d (n=%d) alone differs from the oracle" % (i, len(arr))
        assert np.array_equal(mixed[i], alone[i]), "request %d (n=%d) differs in the mix" % (i, len(arr))


def test_server_result_equals_packed_sort_of_one_array():
    import torch
    dtype = bs.I32_I32
    reqs = make_requests(dtype, 24, seed=99, max_len=8192)
    with bs.Server(dtype, budget_bytes=64 << 20) as srv:
        served = sort_in_mix(srv, dtype, reqs)
    for arr, got in zip(reqs, served):
        d = to_device(arr)
        out = empty_device(arr.nbytes)
        bs.sort_packed(dtype, d.data_ptr(), out.data_ptr(), len(arr), 1, 0, None,
                       torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(from_device(out[:arr.nbytes], bs.NP_DTYPES[dtype]), got)


def test_host_memory_requests_pinned_and_pageable():
    import torch
    dtype = bs.I32_I32
    reqs = make_requests(dtype, 40, seed=5, max_len=20000)
    with bs.Server(dtype, budget_bytes=64 << 20) as srv:
        tickets, outs = [], []
        for i, arr in enumerate(reqs):
            if i % 2:
                src = torch.from_numpy(arr.view(np.uint8).copy()).pin_memory()
                dst = torch.empty_like(src).pin_memory()
                sp, dp = src.data_ptr(), dst.data_ptr()
                keep = (src, dst)
            else:
                src = arr.copy()
                dst = np.empty_like(arr)
                sp, dp = src.ctypes.data, dst.ctypes.data
                keep = (src, dst)
            tickets.append(srv.submit(sp, dp, len(arr), bs.MEM_HOST))
            outs.append(keep)
        for t in tickets:
            assert srv.wait(t, 60_000_000) == bs.OK
    for arr, (_, dst) in zip(reqs, outs):
        got = dst.numpy().view(bs.NP_DTYPES[dtype]) if isinstance(dst, torch.Tensor) else dst
        assert np.array_equal(got, expected_one(dtype, 0, arr))


def test_budget_bounds_the_arena_and_rejects_oversized_requests():
    import torch
    dtype = bs.I32_I32
    budget = 1 << 20                                        # 1 MiB: two 65536-record requests
    rng = np.random.default_rng(3)
    reqs = [workloads.make_packed(dtype, 65536, 1, "uniform", seed=int(s)) for s in rng.integers(0, 1 << 30, 8)]
    with bs.Server(dtype, budget_bytes=budget, max_inflight=8) as srv:
        outs = sort_in_mix(srv, dtype, reqs, threads=1)
        s = srv.stats()
        assert s.arena_bytes == budget and 0 < s.peak_arena_bytes <= budget
        big = empty_device(2 << 20)
        st, _ = srv.submit_status(big.data_ptr(), big.data_ptr(), bs.ragged_max_length(dtype) + 1)
        assert st == 2                                      # beyond the longest sortable array
        torch.cuda.synchronize()
    with bs.Server(dtype, budget_bytes=256 << 10) as small:  # 256 KiB < one 65536-record request
        st, _ = small.submit_status(big.data_ptr(), big.data_ptr(), 65536)
        assert st == bs.ERR_BUDGET
        assert small.stats().rejected == 1
    for arr, got in zip(reqs, outs):
        assert np.array_equal(got, expected_one(dtype, 0, arr))


def test_zero_length_and_queue_state():
    dtype = bs.I32
    with bs.Server(dtype, budget_bytes=1 << 20) as srv:
        t = srv.submit(0, 0, 0)
        assert srv.poll(t)[0] == bs.REQ_DONE
        assert srv.wait(t, 60_000_000) == bs.OK
        srv.drain(5_000_000)
        assert srv.stats().queued == 0
