"""Integer-shift FDR (src/intfdr.jl) over the C ABI."""
from __future__ import annotations

import ctypes as C
from fractions import Fraction

import numpy as np
import torch

from . import _lib
from .arrays import as_device_f32, fortran_empty, ptr, stream_handle


def _rate_mode(rates):
    """FDR_RATES_F32 when the rates are float32 values (Julia Float32 arithmetic), else
    FDR_RATES_F64."""
    if isinstance(rates, np.ndarray) and rates.dtype == np.float32:
        return _lib.FDR_RATES_F32
    if isinstance(rates, torch.Tensor) and rates.dtype == torch.float32:
        return _lib.FDR_RATES_F32
    if isinstance(rates, (np.float32,)):
        return _lib.FDR_RATES_F32
    return _lib.FDR_RATES_F64


def _shifts_exact(rates, Nt):
    """round(rate*t) (ties to even) in exact rational arithmetic, for Fraction rates."""
    out = []
    for r in rates:
        for t in range(Nt):
            v = Fraction(r) * t
            fl = v.numerator // v.denominator
            d = v - fl
            if d > Fraction(1, 2) or (d == Fraction(1, 2) and fl % 2 != 0):
                fl += 1
            out.append(fl)
    return out


def intshift_(dout, din, rate, stream=None):
    """intshift! (intfdr.jl:7-14)."""
    din = as_device_f32(din)
    mode = _rate_mode(rate)
    _lib.check(_lib.lib().fdr_intshift(ptr(din), din.shape[0], din.shape[1], float(rate), mode,
                                       ptr(dout), stream_handle(stream)))
    return dout


def intshift(din, rate, stream=None):
    """intshift (intfdr.jl:23-26)."""
    din = as_device_f32(din)
    dout = fortran_empty(*din.shape)
    return intshift_(dout, din, rate, stream)


def intfdr_(fdr, spectrogram, rates, stream=None):
    """intfdr! (intfdr.jl:34-45).  ``rates``: a sequence of numbers (float64 arithmetic),
    a float32 array (float32 arithmetic) or Fractions (exact rational arithmetic, as
    Julia's Rational ranges from batchrates)."""
    spec = as_device_f32(spectrogram)
    Nf, Nt = spec.shape
    rl = list(rates) if not isinstance(rates, (np.ndarray, torch.Tensor)) else rates
    Nr = len(rl)
    if tuple(fdr.shape) != (Nf, Nr):
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT, "fdr has the wrong size")
    if Nr and isinstance(rl, list) and any(isinstance(r, Fraction) for r in rl):
        sh = _shifts_exact(rl, Nt)
        arr = (C.c_int64 * len(sh))(*sh)
        _lib.check(_lib.lib().fdr_intfdr_shifts(ptr(spec), Nf, Nt, arr, Nr, ptr(fdr),
                                                stream_handle(stream)))
        return fdr
    mode = _rate_mode(rates)
    vals = np.asarray(rl.cpu().numpy() if isinstance(rl, torch.Tensor) else rl, dtype=np.float64)
    arr = (C.c_double * max(1, Nr))(*vals.tolist())
    _lib.check(_lib.lib().fdr_intfdr(ptr(spec), Nf, Nt, arr, Nr, mode, ptr(fdr),
                                     stream_handle(stream)))
    return fdr


def intfdr(spectrogram, rates, stream=None):
    """intfdr (intfdr.jl:56-61)."""
    spec = as_device_f32(spectrogram)
    Nr = len(rates)
    fdr = fortran_empty(spec.shape[0], Nr)
    return intfdr_(fdr, spec, rates, stream)
