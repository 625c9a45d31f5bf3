"""Chirp-Z De-Doppler Transform (src/zdtfdr.jl) over the C ABI.

Julia's mutating functions keep their names with a trailing underscore in place of "!":
``input_``, ``preprocess_``, ``convolve_``, ``postprocess_``, ``output_``, ``zdtfdr_``.
"""
from __future__ import annotations

import ctypes as C
from fractions import Fraction

import numpy as np
import torch

from . import _lib
from .arrays import (as_device_f32, complex_matrix_view, fortran_empty, host_hit_buffer, ptr,
                     stream_handle)

_WINDOWS = {"rect": _lib.FDR_WINDOW_RECT, "hamming": _lib.FDR_WINDOW_HAMMING}


def _range_params(rates):
    """(r0, dr, Nr) of an equally spaced sequence of rates (zdtfdr.jl:78-87)."""
    if hasattr(rates, "start") and hasattr(rates, "step") and hasattr(rates, "length"):
        return rates.start, rates.step, int(rates.length)
    if isinstance(rates, range):
        return rates.start, rates.step, len(rates)
    vals = list(rates)
    if not vals:
        raise ValueError("empty rate range")
    if len(vals) == 1:
        return vals[0], 1, 1
    step = vals[1] - vals[0]
    return vals[0], step, len(vals)


class ZDTWorkspace:
    """ZDTWorkspace (zdtfdr.jl:10-87): owns F, Y (with Yf/Ys views), V and FFT scratch on
    the device.  Construct from a spectrogram and either a rate range or (r0, dr, Nr)::

        ws = ZDTWorkspace(spec, rates)                  # rates: range-like
        ws = ZDTWorkspace(spec, r0, dr, Nr, factors=(2, 3, 5))

    ``spectrogram`` may be None to create an empty workspace of size (Nf, Nt) given by
    ``shape``.  Extra keyword flags: ``exact_phase`` (reduce chirp phases exactly instead
    of reproducing the reference's Float32 arguments in the staged stages),
    ``staged_only`` (zdtfdr_ always runs the staged kernels) and ``mixed_precision`` (the
    fused output pass runs its DFTs as split-bfloat16 tensor-core contractions where the
    four-step split has P = 2048, on tcgen05 with tensor-memory accumulators (e.g. Nf = 2^20
    and 2^21 with Nt <= 16), or P = 1024, with mma.sync (e.g. Nf = 2^19); the split is the
    same as without the flag; ~1e-5 relative error instead of ~1e-6) and
    ``fast_stats`` (the snr statistics of ``zdtfdr_protohits_`` come from float64 moments
    accumulated while the FDR is written: two fewer FDR reads, last bits of m and s may
    differ from the reference's Float32 values).
    """

    def __init__(self, spectrogram, r0_or_rates, dr=None, Nr=None, factors=(2, 3, 5), *,
                 output_aligned=False, exact_phase=False, staged_only=False, mixed_precision=False,
                 fast_stats=False, shape=None, stream=None):
        if dr is None:
            r0, dr, Nr = _range_params(r0_or_rates)
        else:
            r0 = r0_or_rates
        if spectrogram is not None:
            spec = as_device_f32(spectrogram)
            Nf, Nt = spec.shape
        else:
            spec = None
            Nf, Nt = shape
        flags = 0
        if output_aligned:
            flags |= _lib.FDR_ZDT_OUTPUT_ALIGNED
        if exact_phase:
            flags |= _lib.FDR_ZDT_EXACT_PHASE
        if staged_only:
            flags |= _lib.FDR_ZDT_STAGED_ONLY
        if mixed_precision:
            flags |= _lib.FDR_ZDT_MIXED_PRECISION
        if fast_stats:
            flags |= _lib.FDR_ZDT_FAST_STATS
        farr, nf = _lib.i64_array([int(f) for f in factors])
        h = C.c_void_p()
        _lib.check(_lib.lib().fdr_zdt_create(
            C.byref(h), ptr(spec), int(Nf), int(Nt), float(np.float32(float(Fraction(r0)))),
            float(np.float32(float(Fraction(dr)))), int(Nr), farr, nf, flags,
            stream_handle(stream)))
        self._h = h
        self.factors = tuple(int(f) for f in factors)
        info = _lib.fdr_zdt_info()
        _lib.check(_lib.lib().fdr_zdt_get_info(self._h, C.byref(info)))
        self._info = info

    # -- lifecycle ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().fdr_zdt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- fields (zdtfdr.jl:10-35) -------------------------------------------------------
    Nf = property(lambda self: int(self._info.Nf))
    Nt = property(lambda self: int(self._info.Nt))
    Nr = property(lambda self: int(self._info.Nr))
    Nl = property(lambda self: int(self._info.Nl))
    K = property(lambda self: int(self._info.K))
    r0 = property(lambda self: float(self._info.r0))
    dr = property(lambda self: float(self._info.dr))
    fused = property(lambda self: bool(self._info.fused))

    def _buffers(self):
        F, Y, V = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _lib.check(_lib.lib().fdr_zdt_buffers(self._h, C.byref(F), C.byref(Y), C.byref(V)))
        return F.value, Y.value, V.value

    @property
    def F(self):
        return complex_matrix_view(self._buffers()[0], self.K, self.Nt, self)

    @property
    def Y(self):
        return complex_matrix_view(self._buffers()[1], self.K, self.Nl, self)

    @property
    def Yf(self):
        return self.Y[:, : self.Nt]

    @property
    def Ys(self):
        return self.Y[:, : self.Nr]

    @property
    def V(self):
        return complex_matrix_view(self._buffers()[2], self.K, self.Nl, self)

    def nbytes(self):
        """Base.sizeof(ws) (zdtfdr.jl:101-103): device bytes owned by the workspace."""
        return int(self._info.bytes)

    def __repr__(self):  # Base.show (zdtfdr.jl:89-99)
        return (f"ZDTWorkspace(Nf={self.Nf},Nt={self.Nt},r0={self.r0},δr={self.dr},"
                f"Nr={self.Nr},Nl={self.Nl},{self.factors})")

    # -- timing ---------------------------------------------------------------------
    def set_timing(self, enable=True):
        _lib.check(_lib.lib().fdr_zdt_set_timing(self._h, 1 if enable else 0))

    def stage_times(self):
        times = (C.c_float * 64)()
        names = (C.c_char_p * 64)()
        n = C.c_int()
        _lib.check(_lib.lib().fdr_zdt_stage_times(self._h, times, 64, C.byref(n), names))
        return [(names[i].decode(), float(times[i])) for i in range(n.value)]


def fused_split(Nf, Nt, Nr, *, mixed_precision=False, staged_only=False):
    """The four-step split (P, Q), Nf = P * Q, that the fused path of a workspace with these
    sizes and flags uses (P residues in the input and output passes, Q bins per czt CTA),
    or None when zdtfdr_ runs the staged kernels.  Host arithmetic only."""
    flags = (_lib.FDR_ZDT_MIXED_PRECISION if mixed_precision else 0) | (
        _lib.FDR_ZDT_STAGED_ONLY if staged_only else 0)
    P, Q = C.c_int64(0), C.c_int64(0)
    st = _lib.lib().fdr_zdt_fused_split(int(Nf), int(Nt), int(Nr), flags, C.byref(P), C.byref(Q))
    if st == _lib.FDR_ERR_UNSUPPORTED_SIZE:
        return None
    _lib.check(st)
    return int(P.value), int(Q.value)


def _window_args(w, K, Nf):
    if w is None or w == "rect":
        return _lib.FDR_WINDOW_RECT, None
    if isinstance(w, str):
        if w not in _WINDOWS:
            raise _lib.FDRError(_lib.FDR_ERR_UNSUPPORTED_WINDOW, f"unsupported window type ({w})")
        return _WINDOWS[w], None
    if callable(w):
        vals = torch.tensor([float(w(n, Nf)) for n in range(K)], dtype=torch.float64,
                            device="cuda")
        return _lib.FDR_WINDOW_CUSTOM, vals
    raise _lib.FDRError(_lib.FDR_ERR_UNSUPPORTED_WINDOW, f"unsupported window type ({w})")


def input_(ws: ZDTWorkspace, spectrogram, stream=None):
    """input! (zdtfdr.jl:209-212)."""
    spec = as_device_f32(spectrogram)
    _check_spec(ws, spec)
    _lib.check(_lib.lib().fdr_zdt_input(ws._h, ptr(spec), stream_handle(stream)))


def preprocess_(ws: ZDTWorkspace, r0=None, stream=None):
    """preprocess! (zdtfdr.jl:221-239)."""
    r0 = ws.r0 if r0 is None else float(np.float32(float(r0)))
    _lib.check(_lib.lib().fdr_zdt_preprocess(ws._h, r0, stream_handle(stream)))


def convolve_(ws: ZDTWorkspace, stream=None):
    """convolve! (zdtfdr.jl:249-253)."""
    _lib.check(_lib.lib().fdr_zdt_convolve(ws._h, stream_handle(stream)))


def postprocess_(ws: ZDTWorkspace, w="rect", stream=None):
    """postprocess! (zdtfdr.jl:297-321); w is "rect", "hamming" or f(k, Nf)."""
    code, vals = _window_args(w, ws.K, ws.Nf)
    _lib.check(_lib.lib().fdr_zdt_postprocess(ws._h, code, ptr(vals), stream_handle(stream)))
    if vals is not None:
        torch.cuda.current_stream().synchronize()


def output_(dest, ws: ZDTWorkspace, stream=None):
    """output! (zdtfdr.jl:328-331): dest (Nf x Nr) = irfft(Ys)."""
    _check_dest(ws, dest)
    _lib.check(_lib.lib().fdr_zdt_output(ws._h, ptr(dest), stream_handle(stream)))
    return dest


def _check_spec(ws, spec):
    if tuple(spec.shape) != (ws.Nf, ws.Nt):
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT,
                            f"spectrogram size {tuple(spec.shape)} != ({ws.Nf}, {ws.Nt})")


def _check_dest(ws, dest):
    from .arrays import is_fortran
    if (not isinstance(dest, torch.Tensor) or dest.dtype != torch.float32
            or dest.device.type != "cuda" or tuple(dest.shape) != (ws.Nf, ws.Nr)
            or not is_fortran(dest)):
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT,
                            f"dest must be a column-major float32 CUDA ({ws.Nf}, {ws.Nr}) matrix")


def zdtfdr_(dests, ws: ZDTWorkspace, spectrogram=None, *, r0=None, w="rect", stream=None):
    """zdtfdr!([w,] dests, ws[, spectrogram]; r0) (zdtfdr.jl:349-378).

    ``dests`` is one (Nf, Nr) matrix or a sequence of them; ``r0`` is a scalar or a sequence
    cycled over ``dests`` (Iterators.cycle, zdtfdr.jl:354).  Returns ``dests``.
    """
    single = isinstance(dests, torch.Tensor)
    dl = [dests] if single else list(dests)
    for d in dl:
        _check_dest(ws, d)
    if r0 is None:
        r0s = [ws.r0] * len(dl)
    elif np.ndim(r0) == 0 and not isinstance(r0, (list, tuple)):
        r0s = [float(np.float32(float(r0)))] * len(dl)
    else:
        rl = [float(np.float32(float(x))) for x in r0]
        r0s = [rl[i % len(rl)] for i in range(len(dl))]
    spec = None
    if spectrogram is not None:
        spec = as_device_f32(spectrogram)
        _check_spec(ws, spec)
    code, vals = _window_args(w, ws.K, ws.Nf)
    n = len(dl)
    r0_arr = (C.c_float * max(1, n))(*r0s)
    d_arr = (C.c_void_p * max(1, n))(*[d.data_ptr() for d in dl])
    _lib.check(_lib.lib().fdr_zdt_execute(ws._h, ptr(spec), r0_arr, n, d_arr, code, ptr(vals),
                                          stream_handle(stream)))
    if vals is not None:
        torch.cuda.current_stream().synchronize()
    return dests


def zdtfdr_nodest_(ws: ZDTWorkspace, spectrogram=None, *, r0=None, w="rect", stream=None):
    """zdtfdr!([w,] ws[, spectrogram]; r0) with no dest (zdtfdr.jl:382-396): the result is
    left in ws.Ys (before the output FFT)."""
    if spectrogram is not None:
        input_(ws, spectrogram, stream)
    preprocess_(ws, r0, stream)
    convolve_(ws, stream)
    postprocess_(ws, w, stream)
    return None


def zdtfdr(ws: ZDTWorkspace, spectrogram=None, *, r0=None, w="rect", stream=None):
    """zdtfdr([w,] ws[, spectrogram]; r0) (zdtfdr.jl:412-421): allocates the (Nf, Nr)
    float32 dest on the device."""
    dest = fortran_empty(ws.Nf, ws.Nr)
    zdtfdr_(dest, ws, spectrogram, r0=r0, w=w, stream=stream)
    return dest


def zdtfdr_protohits_(dests, ws: ZDTWorkspace, spectrogram=None, *, r0=None, w="rect",
                      threshold=10.0, snr=True, capacity=None, stream=None,
                      return_threshold=False):
    """zdtfdr!(dests, ws[, spectrogram]; r0) followed by findprotohits(dests, threshold; snr)
    with the fused threshold/proto-hit scan of the library (fdr_zdtfdr_protohits): with
    ``snr`` the statistics are fdrstats's Float32 pairwise values over the dests (or, for a
    workspace made with ``fast_stats=True``, float64 moments accumulated while the FDR is
    written), and the threshold's type follows ``threshold`` as in findprotohits.  Returns
    an int64 numpy array of zero-based (i, j) hits in column-major order (j offset by b*Nr
    for the b-th dest)."""
    single = isinstance(dests, torch.Tensor)
    dl = [dests] if single else list(dests)
    for d in dl:
        _check_dest(ws, d)
    if r0 is None:
        r0s = [ws.r0] * len(dl)
    elif np.ndim(r0) == 0 and not isinstance(r0, (list, tuple)):
        r0s = [float(np.float32(float(r0)))] * len(dl)
    else:
        rl = [float(np.float32(float(x))) for x in r0]
        r0s = [rl[i % len(rl)] for i in range(len(dl))]
    spec = None
    if spectrogram is not None:
        spec = as_device_f32(spectrogram)
        _check_spec(ws, spec)
    code, vals = _window_args(w, ws.K, ws.Nf)
    n = len(dl)
    r0_arr = (C.c_float * n)(*r0s)
    d_arr = (C.c_void_p * n)(*[d.data_ptr() for d in dl])
    cap = (1 << 20) if capacity is None else int(capacity)
    hits = host_hit_buffer(cap)
    count, thr = C.c_int64(), C.c_double()
    st = _lib.lib().fdr_zdtfdr_protohits(ws._h, ptr(spec), r0_arr, n, d_arr, code, ptr(vals),
                                         float(threshold), _lib.snr_mode(threshold, snr),
                                         ptr(hits), cap,
                                         C.byref(count), C.byref(thr), stream_handle(stream))
    if vals is not None:
        torch.cuda.current_stream().synchronize()
    if st == _lib.FDR_ERR_CAPACITY:
        # the FDR and the threshold are computed: collect the hits with a large enough buffer
        from .fdrutils import findprotohits
        out = findprotohits(dl, thr.value, snr=False, capacity=int(count.value), stream=stream)
        return (out, thr.value) if return_threshold else out
    _lib.check(st)
    out = hits[: count.value].numpy().copy()
    return (out, thr.value) if return_threshold else out


def _blocks_args(ws, dest, blocks):
    bl = [int(b) for b in np.asarray(blocks).ravel()]
    if not bl:
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT, "need at least one rate block")
    from .arrays import is_fortran
    if (not isinstance(dest, torch.Tensor) or dest.dtype != torch.float32
            or dest.device.type != "cuda" or tuple(dest.shape) != (ws.Nf, 8 * len(bl))
            or not is_fortran(dest)):
        raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT,
                            f"dest must be a column-major float32 CUDA ({ws.Nf}, {8 * len(bl)}) matrix")
    return (C.c_int32 * len(bl))(*bl), len(bl)


def zdtfdr_blocks_(dest, ws: ZDTWorkspace, spectrogram, blocks, *, w="rect", stream=None):
    """zdtfdr! over the 8-rate blocks ``blocks`` of the workspace's rate grid in one pass
    (fdr_zdt_execute_blocks): FDR column 8i+u of ``dest`` is rate r0 + (8*blocks[i]+u)*dr."""
    barr, nb = _blocks_args(ws, dest, blocks)
    spec = None
    if spectrogram is not None:
        spec = as_device_f32(spectrogram)
        _check_spec(ws, spec)
    code, vals = _window_args(w, ws.K, ws.Nf)
    _lib.check(_lib.lib().fdr_zdt_execute_blocks(ws._h, ptr(spec), barr, nb, ptr(dest), code,
                                                 ptr(vals), stream_handle(stream)))
    if vals is not None:
        torch.cuda.current_stream().synchronize()
    return dest


def zdtfdr_blocks_protohits_(dest, ws: ZDTWorkspace, spectrogram, blocks, *, w="rect",
                             threshold=10.0, snr=True, capacity=None, stream=None,
                             return_threshold=False):
    """zdtfdr_blocks_ followed by the fused proto-hit scan of ``dest``
    (fdr_zdtfdr_blocks_protohits); hits are zero-based (i, dest column) pairs."""
    barr, nb = _blocks_args(ws, dest, blocks)
    spec = None
    if spectrogram is not None:
        spec = as_device_f32(spectrogram)
        _check_spec(ws, spec)
    code, vals = _window_args(w, ws.K, ws.Nf)
    cap = (1 << 20) if capacity is None else int(capacity)
    hits = host_hit_buffer(cap)
    count, thr = C.c_int64(), C.c_double()
    st = _lib.lib().fdr_zdtfdr_blocks_protohits(ws._h, ptr(spec), barr, nb, ptr(dest), code,
                                                ptr(vals), float(threshold),
                                                _lib.snr_mode(threshold, snr),
                                                ptr(hits), cap, C.byref(count), C.byref(thr),
                                                stream_handle(stream))
    if vals is not None:
        torch.cuda.current_stream().synchronize()
    if st == _lib.FDR_ERR_CAPACITY:
        from .fdrutils import findprotohits
        out = findprotohits(dest, thr.value, snr=False, capacity=int(count.value), stream=stream)
        return (out, thr.value) if return_threshold else out
    _lib.check(st)
    out = hits[: count.value].numpy().copy()
    return (out, thr.value) if return_threshold else out
