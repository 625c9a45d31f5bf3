"""Device-array plumbing between torch CUDA tensors and the C ABI.

Matrices follow the reference's Julia column-major layout.  A logical (Nf, Nt) matrix is a
torch tensor of shape (Nf, Nt) with strides (1, Nf) ("Fortran order"); indexing
``m[n, t]`` addresses the same element as Julia's ``m[n+1, t+1]``.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import torch


def stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


_hit_buffers = threading.local()


def host_hit_buffer(capacity: int) -> torch.Tensor:
    """An int64 hit buffer of at least (capacity, 2) in pinned host memory, kept per host
    thread and reused by the next call (callers copy the hits out before returning).
    Pinned memory is mapped into the device's address space, so the library's kernels write
    the hits into it directly: reading them needs no device-to-host copy, which would go
    through a copy engine and wait behind an unrelated host-to-device transfer in flight (the
    next spectrogram of a pipeline)."""
    cap = max(1, int(capacity))
    buf = getattr(_hit_buffers, "buf", None)
    if buf is None or buf.shape[0] < cap:
        buf = torch.empty((cap, 2), dtype=torch.int64, pin_memory=True)
        _hit_buffers.buf = buf
    return buf


def is_fortran(t: torch.Tensor) -> bool:
    if t.dim() == 1:
        return t.stride(0) == 1
    if t.dim() != 2:
        return False
    n0, n1 = t.shape
    return (t.stride(0) == 1 or n0 <= 1) and (t.stride(1) == n0 or n1 <= 1)


def fortran_empty(rows, cols, dtype=torch.float32, device="cuda"):
    return torch.empty((cols, rows), dtype=dtype, device=device).t()


def fortran_zeros(rows, cols, dtype=torch.float32, device="cuda"):
    return torch.zeros((cols, rows), dtype=dtype, device=device).t()


def as_device_f32(x, device="cuda") -> torch.Tensor:
    """A float32 CUDA tensor in column-major layout (copies only when needed)."""
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32))
    if not isinstance(x, torch.Tensor):
        x = torch.as_tensor(x, dtype=torch.float32)
    if x.dtype != torch.float32:
        raise TypeError("the FDR library implements Float32 spectrograms and FDR matrices only")
    if x.device.type != "cuda":
        x = x.to(device)
    if x.dim() == 1:
        return x.contiguous()
    if not is_fortran(x):
        x = x.t().contiguous().t()
    return x


def ptr(t) -> C.c_void_p:
    if t is None:
        return C.c_void_p(None)
    return C.c_void_p(t.data_ptr())


class _DeviceView:
    """__cuda_array_interface__ wrapper over memory owned by a library workspace."""

    def __init__(self, address, shape, typestr, strides_bytes, owner):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape),
            "typestr": typestr,
            "data": (int(address), False),
            "strides": tuple(strides_bytes),
            "version": 3,
        }
        self._owner = owner


def complex_matrix_view(address, rows, cols, owner) -> torch.Tensor:
    """(rows, cols) complex64 column-major view of library-owned device memory."""
    v = _DeviceView(address, (rows, cols), "<c8", (8, 8 * rows), owner)
    t = torch.as_tensor(v, device="cuda")
    t._fdr_owner = owner  # keep the workspace alive while the view exists
    return t
