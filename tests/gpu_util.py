"""Device-buffer helpers for the GPU tests (torch is only the allocator here)."""
import numpy as np


def to_device(arr):
    import torch
    flat = np.ascontiguousarray(arr).view(np.uint8)
    return torch.from_numpy(flat.copy()).cuda()


def from_device(t, np_dtype):
    return t.cpu().numpy().view(np_dtype)


def empty_device(nbytes):
    import torch
    return torch.empty(max(nbytes, 16), dtype=torch.uint8, device="cuda")


def stream_handle():
    import torch
    return torch.cuda.current_stream().cuda_stream
