"""Argument checking for the drop-in module: host (numpy) and device (torch CUDA)
arrays, with the reference binding's error types.

The reference declares its arrays as nanobind ndarrays of a fixed dtype and
device (src/bindings.cpp:27-35); a mismatching array is rejected with
TypeError there, and so here.  Unlike the reference, which reads `.data()` as
if dense (its ndarray types carry no contiguity constraint), non-contiguous
device arrays are rejected with ValueError and host arrays are copied to a
dense layout.
"""
from __future__ import annotations

import numpy as np

try:  # torch is the device-buffer provider; it is required for device arrays.
    import torch
except ImportError:  # pragma: no cover - torch is part of the supported image
    torch = None


def host_array(a, dtype, name: str, ndim: int = 1) -> np.ndarray:
    """A dense host array of exactly `dtype` (TypeError otherwise)."""
    if torch is not None and isinstance(a, torch.Tensor):
        if a.device.type != "cpu":
            raise TypeError(f"{name}: expected a host (CPU) array, got device {a.device}")
        a = a.numpy()
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{name}: expected a numpy.ndarray of {np.dtype(dtype).name}, "
                        f"got {type(a).__name__}")
    if a.dtype != np.dtype(dtype):
        raise TypeError(f"{name}: expected dtype {np.dtype(dtype).name}, got {a.dtype}")
    if a.ndim != ndim:
        raise TypeError(f"{name}: expected {ndim}-D array, got {a.ndim}-D")
    return np.ascontiguousarray(a)


_TORCH_DTYPES = {}
if torch is not None:
    _TORCH_DTYPES = {"float64": torch.float64, "float32": torch.float32}


def device_array(a, dtype: str, name: str, ndim: int = 1):
    """A contiguous CUDA tensor of `dtype` viewing the caller's memory (zero copy)."""
    if torch is None:
        raise TypeError(f"{name}: torch is required for device arrays")
    t = a
    if not isinstance(t, torch.Tensor):
        if hasattr(a, "__dlpack__"):
            t = torch.from_dlpack(a)
        elif hasattr(a, "__cuda_array_interface__"):
            t = torch.as_tensor(a, device="cuda")
        else:
            raise TypeError(f"{name}: expected a CUDA array (torch.Tensor, DLPack or "
                            f"__cuda_array_interface__), got {type(a).__name__}")
    if t.device.type != "cuda":
        raise TypeError(f"{name}: expected a CUDA array, got device {t.device}")
    if t.dtype != _TORCH_DTYPES[dtype]:
        raise TypeError(f"{name}: expected dtype {dtype}, got {t.dtype}")
    if t.dim() != ndim:
        raise TypeError(f"{name}: expected {ndim}-D array, got {t.dim()}-D")
    if not t.is_contiguous():
        raise ValueError(f"{name}: array must be contiguous (C order)")
    return t


def stream_of(t) -> int:
    """cudaStream_t (as int) of torch's current stream on t's device."""
    return torch.cuda.current_stream(t.device).cuda_stream
