"""The PyTorch operators torch.ops.b200sort.sort_ragged / sort_packed
(cuda-sort_b200/b200sort_torch.py).  CPU: registration, schema, shape
inference under fake tensors, and the loud refusal of CPU tensors and bad
layouts.  GPU: the operators' outputs against the oracle, default and stable
modes, every element layout, on the current stream."""
import numpy as np
import pytest
import torch

import b200sort as bs
import b200sort_torch  # noqa: F401  (registers the operators)
import cpu_oracle as orc
import workloads


def test_operators_are_registered_with_their_schema():
    assert "sort_ragged" in dir(torch.ops.b200sort) and "sort_packed" in dir(torch.ops.b200sort)
    schema = str(torch.ops.b200sort.sort_ragged.default._schema)
    assert "Tensor values" in schema and "Tensor offsets" in schema and "bool stable" in schema


def test_shape_inference_under_fake_tensors():
    from torch._subclasses.fake_tensor import FakeTensorMode
    with FakeTensorMode():
        v = torch.empty(1000, 2, dtype=torch.int32, device="cuda")
        o = torch.empty(11, dtype=torch.int64, device="cuda")
        out = torch.ops.b200sort.sort_ragged(v, o, True)
        assert out.shape == (1000, 2) and out.dtype == torch.int32
        out = torch.ops.b200sort.sort_packed(v, 100)
        assert out.shape == (1000, 2)


def test_cpu_tensors_and_bad_layouts_are_refused():
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        torch.ops.b200sort.sort_ragged(torch.zeros(8, dtype=torch.int32), torch.tensor([0, 8]))
    with pytest.raises(TypeError):
        b200sort_torch._dtype_of(torch.zeros(8, 3, dtype=torch.int32))
    with pytest.raises(TypeError):
        b200sort_torch._dtype_of(torch.zeros(8, dtype=torch.float32))


def _expected(dtype, flags, data, off):
    mode = orc.MODE_STABLE if flags else (orc.MODE_NETWORK if dtype in (bs.I32_I32, bs.U64_I32) else orc.MODE_STD)
    return orc.sort_ragged(dtype, data, off, mode, threads=8)


def _as_tensor(dtype, data):
    raw = torch.from_numpy(data.view(np.uint8).copy())
    if dtype == bs.I32:
        return raw.view(torch.int32).cuda()
    if dtype == bs.I32_I32:
        return raw.view(torch.int32).view(-1, 2).cuda()
    if dtype == bs.U64:
        return raw.view(torch.int64).cuda()
    return raw.view(torch.int32).view(-1, 4).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,stable", [(bs.I32, False), (bs.I32_I32, False), (bs.I32_I32, True),
                                          (bs.U64, False), (bs.U64_I32, False), (bs.U64_I32, True)])
def test_sort_ragged_operator_matches_the_oracle(dtype, stable):
    lengths = workloads.ragged_lengths(3000, max_len=20000, seed=9)
    lengths[::17] = 0
    data, off = workloads.make_ragged(dtype, lengths, "distinct16", seed=9, extremes=True)
    v = _as_tensor(dtype, data)
    for off_dtype in (torch.int64, torch.int32):
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            out = torch.ops.b200sort.sort_ragged(v, torch.from_numpy(off).to(off_dtype).cuda(), stable)
        s.synchronize()
        got = out.cpu().numpy().reshape(-1).view(np.uint8).view(bs.NP_DTYPES[dtype])
        assert np.array_equal(got, _expected(dtype, stable, data, off))
    with pytest.raises(RuntimeError, match="offsets"):
        bad = torch.from_numpy(off[::-1].copy()).cuda()
        torch.ops.b200sort.sort_ragged(v, bad)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [bs.I32, bs.I32_I32, bs.U64, bs.U64_I32])
def test_sort_packed_operator_matches_the_oracle(dtype):
    n, arrays = 1000, 300
    data = workloads.make_packed(dtype, n, arrays, "distinct16", seed=4, extremes=True)
    out = torch.ops.b200sort.sort_packed(_as_tensor(dtype, data), n)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(-1).view(np.uint8).view(bs.NP_DTYPES[dtype])
    off = np.arange(arrays + 1, dtype=np.int64) * n
    assert np.array_equal(got, _expected(dtype, False, data, off))
