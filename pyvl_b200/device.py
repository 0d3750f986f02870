"""PyTorch plumbing for the C ABI: device tensors, raw pointers, streams, workspaces.

PyTorch only moves memory here; every computation is a kernel of libpvl_b200.so.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch


def require_cuda() -> torch.device:
    """Return the current CUDA device or raise: the hot path has no CPU fallback."""
    if not torch.cuda.is_available():
        raise RuntimeError("pyvl_b200 runs its kernels on a CUDA GPU (B200); no GPU is available")
    return torch.device("cuda", torch.cuda.current_device())


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_cur_device = getattr(torch._C, "_cuda_getDevice", None)


def stream_ptr(stream: torch.cuda.Stream | None = None) -> int:
    """The stream handle as an integer for a void* argument (the current stream by default;
    read through torch's raw-stream query, which costs far less per call than building a
    Stream object: a step makes dozens of these calls)."""
    if stream is not None:
        return stream.cuda_stream
    if _raw_stream is not None and _cur_device is not None:
        return _raw_stream(_cur_device())
    return torch.cuda.current_stream().cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    """Device address of a tensor as an integer for a void* argument (None -> NULL)."""
    return None if t is None else t.data_ptr()


def to_device(a, dtype=torch.float64, device=None) -> torch.Tensor:
    """Contiguous device tensor of `dtype` (no copy when already one)."""
    dev = device or require_cuda()
    if isinstance(a, torch.Tensor):
        t = a.to(device=dev, dtype=dtype)
        return t.contiguous()
    arr = np.ascontiguousarray(a)
    return torch.from_numpy(arr).to(device=dev, dtype=dtype, non_blocking=False).contiguous()


def to_device_u32(a, device=None) -> torch.Tensor:
    """uint32 host array -> int32 device tensor with the same bit pattern."""
    dev = device or require_cuda()
    arr = np.ascontiguousarray(np.asarray(a, np.uint32)).view(np.int32)
    return torch.from_numpy(arr.copy()).to(dev)


class Workspace:
    """Grow-only device scratch buffer, one per (device, stream)."""

    _pool: dict = {}

    @classmethod
    def get(cls, nbytes: int, stream: torch.cuda.Stream | None = None) -> tuple[ctypes.c_void_p, int]:
        dev = require_cuda()
        s = stream if stream is not None else torch.cuda.current_stream()
        key = (dev.index, s.cuda_stream)
        buf = cls._pool.get(key)
        nbytes = max(int(nbytes), 256)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(int(nbytes * 1.25) + 256, dtype=torch.uint8, device=dev)
            cls._pool[key] = buf
        return ctypes.c_void_p(buf.data_ptr()), buf.numel()

    @classmethod
    def clear(cls) -> None:
        cls._pool.clear()
