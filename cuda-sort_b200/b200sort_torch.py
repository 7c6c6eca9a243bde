"""PyTorch operators over the b200sort C ABI (torch.library custom ops).

    import b200sort_torch            # registers torch.ops.b200sort.*
    out = torch.ops.b200sort.sort_ragged(values, offsets, stable=False)
    out = torch.ops.b200sort.sort_packed(values, n, stable=False)

sort_ragged sorts every array [offsets[a], offsets[a+1]) of a CSR batch
(the reference's partition sort over CSR ranges, SortPartitionsAdaptive_
outofplace, cusort.hpp:2309-2352) and sort_packed every array of a packed
batch (array a at [a*n, a*n + n), the reference's batched one-CTA-per-array
sort, bench.cu:389-393).  Both return a new tensor and run on the current
CUDA stream of the values' device.  Element layouts (values):

  int32, shape (N,)         int32 keys                               B200S_I32
  int32, shape (N, 2)       IntAndData records {key, payload}        B200S_I32_I32
  uint64 or int64, (N,)     uint64 keys (int64 holds the bit pattern; B200S_U64
                            the order is that of the unsigned values)
  int32, shape (N, 4)       {uint64 key (low, high word), payload,   B200S_U64_I32
                            reserved} records

Records compare by key; in the default mode equal keys end in the
reference's network order, with stable=True in input order.  offsets: int32
or int64, arrays + 1 non-decreasing entries from 0 to N, on the same device.
There is no CPU implementation: the operators require CUDA tensors and the
built library, and raise otherwise.
"""
import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import b200sort as bs  # noqa: E402


def _dtype_of(values):
    if values.dtype == torch.int32 and values.dim() == 1:
        return bs.I32
    if values.dtype == torch.int32 and values.dim() == 2 and values.shape[1] == 2:
        return bs.I32_I32
    if values.dtype in (torch.int64, torch.uint64) and values.dim() == 1:
        return bs.U64
    if values.dtype == torch.int32 and values.dim() == 2 and values.shape[1] == 4:
        return bs.U64_I32
    raise TypeError("b200sort: values must be int32 (N,), int32 (N, 2), int64/uint64 (N,) or int32 (N, 4); got %s %s"
                    % (values.dtype, tuple(values.shape)))


def _check_cuda(values):
    if not values.is_cuda:
        raise RuntimeError("b200sort: values must be a CUDA tensor (there is no CPU implementation)")
    if not values.is_contiguous():
        raise RuntimeError("b200sort: values must be contiguous")


@torch.library.custom_op("b200sort::sort_ragged", mutates_args=())
def sort_ragged(values: torch.Tensor, offsets: torch.Tensor, stable: bool = False) -> torch.Tensor:
    _check_cuda(values)
    dtype = _dtype_of(values)
    if offsets.dim() != 1 or offsets.dtype not in (torch.int32, torch.int64) or offsets.device != values.device:
        raise RuntimeError("b200sort: offsets must be a 1-D int32/int64 tensor on the values' device")
    arrays = offsets.numel() - 1
    if arrays < 0:
        raise RuntimeError("b200sort: offsets needs at least one entry")
    if values.shape[0] >= 2 ** 31:
        raise RuntimeError("b200sort: ragged batches address elements with int32 offsets")
    # The kernels read elements [offsets[a], offsets[a+1]): offsets outside
    # [0, N] or decreasing would read out of bounds, so they are checked
    # (one device reduction and a read-back).
    n_el = values.shape[0]
    top = bs.ragged_max_length(dtype, bs.STABLE if stable else 0)
    bad = (offsets[0] != 0) | (offsets[-1] != n_el)
    if arrays > 0:
        lengths = offsets[1:] - offsets[:-1]
        bad = bad | (lengths < 0).any() | (lengths > top).any()
    if bool(bad.item()):
        raise RuntimeError("b200sort: offsets must start at 0, end at N = %d and never decrease, and no array may "
                           "be longer than %d" % (n_el, top))
    off = offsets if offsets.dtype == torch.int32 else offsets.to(torch.int32)
    out = torch.empty_like(values)
    if arrays == 0 or values.numel() == 0:
        return out.copy_(values)
    with torch.cuda.device(values.device):
        st = torch.cuda.current_stream(values.device).cuda_stream
        bs.sort_partitions(dtype, values.data_ptr(), out.data_ptr(), off.contiguous().data_ptr(), arrays, 0,
                           bs.STABLE if stable else 0, st)
    return out


@sort_ragged.register_fake
def _(values, offsets, stable=False):
    _dtype_of(values)
    return torch.empty_like(values)


@torch.library.custom_op("b200sort::sort_packed", mutates_args=())
def sort_packed(values: torch.Tensor, n: int, stable: bool = False) -> torch.Tensor:
    _check_cuda(values)
    dtype = _dtype_of(values)
    total = values.shape[0]
    if n <= 0 or total % n:
        raise RuntimeError("b200sort: the batch length %d is not a multiple of n = %d" % (total, n))
    out = torch.empty_like(values)
    if total == 0:
        return out
    with torch.cuda.device(values.device):
        st = torch.cuda.current_stream(values.device).cuda_stream
        bs.sort_packed(dtype, values.data_ptr(), out.data_ptr(), n, total // n, bs.STABLE if stable else 0, None, st)
    return out


@sort_packed.register_fake
def _(values, n, stable=False):
    _dtype_of(values)
    return torch.empty_like(values)
