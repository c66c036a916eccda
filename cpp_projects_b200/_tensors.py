"""Small helpers turning torch tensors into raw device pointers for the C ABI."""
from __future__ import annotations

import ctypes

import torch


def dev_ptr(t: torch.Tensor, dtype: torch.dtype | None = None, name: str = "tensor") -> int:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must live on a CUDA device (got {t.device})")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype} (got {t.dtype})")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t.data_ptr()


def opt_ptr(t, dtype=None, name="tensor"):
    return None if t is None else dev_ptr(t, dtype, name)


def stream_handle(stream: torch.cuda.Stream | None = None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
