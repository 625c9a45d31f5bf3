"""Fourier-shift FDR (src/fftfdr.jl) over the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .arrays import as_device_f32, complex_matrix_view, fortran_empty, ptr, stream_handle


class FFTFDRWorkspace:
    """fftfdr_workspace (fftfdr.jl:39-59): holds rfft(spectrogram) on the device."""

    def __init__(self, spectrogram, bunaligned=True, stream=None):
        spec = as_device_f32(spectrogram)
        self.Nf, self.Nt = (int(x) for x in spec.shape)
        h = C.c_void_p()
        _lib.check(_lib.lib().fdr_fftfdr_workspace(C.byref(h), ptr(spec), self.Nf, self.Nt,
                                                   stream_handle(stream)))
        self._h = h

    @property
    def dest_rfft(self):
        p = C.c_void_p()
        _lib.check(_lib.lib().fdr_fftfdr_rfft_buffer(self._h, C.byref(p)))
        return complex_matrix_view(p.value, self.Nf // 2 + 1, self.Nt, self)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().fdr_fftfdr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fftfdr_workspace(spectrogram, bunaligned=True, stream=None):
    return FFTFDRWorkspace(spectrogram, bunaligned, stream)


def fftfdr_workspace_(ws, spectrogram, bunaligned=True, stream=None):
    """fftfdr_workspace! (fftfdr.jl:69-84); ws None creates a new workspace."""
    if ws is None:
        return FFTFDRWorkspace(spectrogram, bunaligned, stream)
    spec = as_device_f32(spectrogram)
    _lib.check(_lib.lib().fdr_fftfdr_workspace_update(ws._h, ptr(spec), spec.shape[0],
                                                      spec.shape[1], stream_handle(stream)))
    return ws


def _f32(x):
    return float(np.float32(float(x)))


def fdshiftsum_(dest, ws, rate, stream=None):
    """fdshiftsum! (fftfdr.jl:86-96)."""
    _lib.check(_lib.lib().fdr_fdshiftsum(ws._h, _f32(rate), ptr(dest), stream_handle(stream)))
    return dest


def fdshiftsum(ws, rate, stream=None):
    import torch
    dest = torch.empty(ws.Nf, dtype=torch.float32, device="cuda")
    return fdshiftsum_(dest, ws, rate, stream)


def fdshift_(dest, ws, rate, stream=None):
    """fdshift! (fftfdr.jl:104-111): de-Dopplered spectrogram."""
    _lib.check(_lib.lib().fdr_fdshift(ws._h, _f32(rate), ptr(dest), stream_handle(stream)))
    return dest


def fdshift(ws, rate, stream=None):
    dest = fortran_empty(ws.Nf, ws.Nt)
    return fdshift_(dest, ws, rate, stream)


def fftfdr_(fdr, ws, rates, stream=None):
    """fftfdr! (fftfdr.jl:126-134)."""
    rl = [_f32(r) for r in rates]
    if tuple(fdr.shape) != (ws.Nf, len(rl)):
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT, "fdr has the wrong size")
    arr = (C.c_float * max(1, len(rl)))(*rl)
    _lib.check(_lib.lib().fdr_fftfdr(ws._h, arr, len(rl), ptr(fdr), stream_handle(stream)))
    return fdr


def fftfdr(ws, rates, stream=None):
    """fftfdr (fftfdr.jl:143-148)."""
    rl = list(rates)
    fdr = fortran_empty(ws.Nf, len(rl))
    return fftfdr_(fdr, ws, rl, stream)
