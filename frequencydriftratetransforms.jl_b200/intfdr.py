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


def taylor_shifts(Nt, d):
    """Channel offsets p_d(t), t < Nt, of the Taylor-tree path of total drift d (Nt a power of
    two): the path of drift floor(|d|/2) over each half, the second half offset by
    ceil(|d|/2), negated for d < 0."""
    if Nt & (Nt - 1) or Nt < 1 or abs(d) > max(Nt - 1, 0):
        raise ValueError("Nt must be a power of two and |d| <= Nt-1")

    def path(L, dd):
        if L == 1:
            return [0]
        half = path(L // 2, dd // 2)
        return half + [(dd + 1) // 2 + x for x in half]

    p = path(Nt, abs(d))
    return [x if d >= 0 else -x for x in p]


def taylorfdr_(fdr, spectrogram, dmin, dmax, stream=None):
    """Taylor-tree integer FDR (fdr_taylor_tree) into ``fdr`` (Nf, dmax-dmin+1): column
    d - dmin sums the spectrogram along the tree path of total drift d, i.e. approximately
    intfdr at rate d/(Nt-1) (exactly for d = 0 and |d| = Nt-1; taylor_shifts gives the
    paths)."""
    spec = as_device_f32(spectrogram)
    Nf, Nt = spec.shape
    if tuple(fdr.shape) != (Nf, dmax - dmin + 1):
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT, "fdr has the wrong size")
    _lib.check(_lib.lib().fdr_taylor_tree(ptr(spec), Nf, Nt, int(dmin), int(dmax), ptr(fdr),
                                          stream_handle(stream)))
    return fdr


def taylorfdr(spectrogram, dmin=None, dmax=None, stream=None):
    """Allocating form of taylorfdr_; the drifts default to -(Nt-1)..Nt-1."""
    spec = as_device_f32(spectrogram)
    Nt = spec.shape[1]
    dmin = -(Nt - 1) if dmin is None else dmin
    dmax = Nt - 1 if dmax is None else dmax
    fdr = fortran_empty(spec.shape[0], dmax - dmin + 1)
    return taylorfdr_(fdr, spec, dmin, dmax, stream)
