"""Host <-> device marshalling shared by the drop-in API.

numpy inputs are copied to the current CUDA device once and results are
copied back (numpy in -> numpy out); torch CUDA tensors are used in place
(torch in -> torch out, on the device).
"""

import numpy as np
import torch

from . import _lib


def device():
    _lib.load()
    return torch.device("cuda", torch.cuda.current_device())


def is_torch(x):
    return isinstance(x, torch.Tensor)


def to_device(x, dtype, contiguous=True):
    """Return (tensor on the current CUDA device, came_from_numpy)."""
    dev = device()
    if is_torch(x):
        t = x.to(device=dev, dtype=dtype)
        return (t.contiguous() if contiguous else t), False
    arr = np.asarray(x)
    t = torch.from_numpy(np.ascontiguousarray(arr, dtype=_np_dtype(dtype)))
    if t.numel():
        t = t.pin_memory() if t.numel() * t.element_size() > (1 << 20) else t
    return t.to(device=dev, non_blocking=True), True


def _np_dtype(dtype):
    return {torch.float64: np.float64, torch.float32: np.float32,
            torch.int32: np.int32, torch.int64: np.int64}[dtype]


def to_output(t, as_numpy):
    if as_numpy:
        return t.cpu().numpy()
    return t


def workspace(nbytes):
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device())
