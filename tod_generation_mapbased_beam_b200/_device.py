"""Device-buffer plumbing shared by the Python entry points: move numpy or
torch inputs into contiguous CUDA tensors of the dtype the C ABI expects, and
hand out the current CUDA stream."""

from __future__ import annotations

import numpy as np
import torch


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError(
            "a CUDA device is required: the TOD kernels run only on the GPU (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def is_tensor(x) -> bool:
    return isinstance(x, torch.Tensor)


def dtype_of(x):
    """numpy dtype of an array-like or tensor."""
    if isinstance(x, torch.Tensor):
        return {torch.float32: np.dtype(np.float32), torch.float64: np.dtype(np.float64),
                torch.int64: np.dtype(np.int64), torch.int32: np.dtype(np.int32)}.get(
                    x.dtype, np.dtype(object))
    return np.asarray(x).dtype


_TORCH = {np.float32: torch.float32, np.float64: torch.float64, np.int64: torch.int64}


def to_device(x, np_dtype, shape=None) -> torch.Tensor:
    """Contiguous CUDA tensor of ``np_dtype`` (copying/converting as needed)."""
    dev = require_cuda()
    tdt = _TORCH[np.dtype(np_dtype).type]
    if isinstance(x, torch.Tensor):
        t = x.to(device=dev, dtype=tdt)
    else:
        a = np.ascontiguousarray(np.asarray(x), dtype=np_dtype)
        t = torch.from_numpy(a).to(dev)
    t = t.contiguous()
    if shape is not None:
        t = t.reshape(shape)
    return t


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()
