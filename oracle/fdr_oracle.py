"""CPU oracle for the FDR transforms -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy/scipy, the algorithms of FrequencyDriftRateTransforms.jl
v0.9.0 on the spectrogram -> frequency-drift-rate (FDR) path.  It is the checker for the
CUDA library: only the tests, the smoke check and the CPU-baseline leg of the benchmark
import it.  The product path (the package's C-ABI library) never calls it.

Two tiers:

* FP32 mirror -- a stage-for-stage restatement of the reference, reproducing its Float32
  argument promotions (e.g. ``Float32(k*l^2) * dr / Nf`` in ``vlow``).  FFTs are scipy's
  pocketfft in single precision where the reference uses FFTW; the reference's FFT library
  is not pinned (Project.toml: "FFTW 1"), so FFT-level parity is pinned only by the
  known answers in test/runtests.jl (3x2 spectrogram) and, beyond that, by the FP64 tier.
* FP64 truth -- circular-shift sums for integer shifts and an exact-phase Fourier-shift sum
  (the fftfdr formulation) in float64 with the phase argument reduced exactly in integer
  arithmetic.

Parity pins: the known answers of test/runtests.jl:5-32 (normalised inverse transforms, as
the reference code computes them) are stored in tests/golden/runtests_known_answers.json
and checked by tests/test_oracle.py.  The Voyager-1 integration data of
test/heavytests.jl:11-14 is not available; a synthetic drifting tone stands in for it.

All arrays are numpy arrays in the reference's layout: a spectrogram of Nf channels by Nt
time steps is an (Nf, Nt) array (frequency fastest in Julia's column-major order; numpy
indexing ``spec[n, t]`` addresses the same element).
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

try:  # scipy's pocketfft keeps float32/complex64 precision and can use threads
    import scipy.fft as _sfft
except Exception:  # pragma: no cover - scipy is present in this image
    _sfft = None


def _fft_mod():
    return _sfft if _sfft is not None else np.fft


# ----------------------------------------------------------------------------------------
# zdtutils.jl
# ----------------------------------------------------------------------------------------

def nextprod(factors, n):
    """Smallest integer >= n whose prime factors are all in ``factors`` (Julia's nextprod)."""
    n = int(n)
    if n <= 1:
        return 1
    best = None
    facs = sorted({int(f) for f in factors})

    def rec(i, cur):
        nonlocal best
        if cur >= n:
            if best is None or cur < best:
                best = cur
            return
        if i == len(facs):
            return
        f = facs[i]
        v = cur
        while True:
            rec(i + 1, v)
            if v >= n:
                break
            v *= f
    rec(0, 1)
    return best


def calcNl(Nt, Nr, factors=(2, 3, 5)):
    """src/zdtutils.jl:7-9 -- nextprod(factors, Nt + Nr - 1)."""
    return nextprod(factors, Nt + Nr - 1)


def growNr(Nt, Nr, factors=(2, 3, 5)):
    """src/zdtutils.jl:17-19 -- calcNl(Nt, Nr, factors) - Nt + 1."""
    return calcNl(Nt, Nr, factors) - Nt + 1


def estimate_memory(Nf, Nt, Nr, Ni=1, No=1, factors=(2, 3, 5)):
    """src/zdtutils.jl:35-53."""
    Nl = calcNl(Nt, Nr, factors)
    Ni += 3
    Nz = 3
    return 4 * ((Nf * Nt) * Ni + (Nf * Nl) * Nz + (Nf * Nr) * No)


def driftrates(r0, dr, Nr):
    """src/zdtutils.jl:62-64 -- range(r0, step=dr, length=Nr) with Float32 r0, dr.

    Julia widens Float32 ranges to twice-precision arithmetic, so element j is the
    correctly rounded Float32 of r0 + j*dr.  Returned as float32 values.
    """
    r0 = float(np.float32(r0))
    dr = float(np.float32(dr))
    return np.array([r0 + j * dr for j in range(Nr)], dtype=np.float64).astype(np.float32)


# ----------------------------------------------------------------------------------------
# batchrates.jl
# ----------------------------------------------------------------------------------------

def _round_nearest_even(x):
    return int(round(x))  # Python rounds half to even, like Julia's RoundNearest


def _round_from_zero(x):
    return int(math.copysign(math.ceil(abs(x)), x)) if x != 0 else 0


def _round_to_zero(x):
    return int(math.trunc(x))


def batchrates(Nt, dhzps, r1, r2=None, Nrb=360):
    """src/batchrates.jl:22-60.  Returns a list of batches; each batch is a list of
    ``Fraction`` drift rates (normalised, channels per time step) with step 1/(Nt-1)."""
    if r2 is None:
        r2 = -r1
    if r2 < r1:
        r1, r2 = r2, r1
    nc1 = _round_nearest_even(r1 / dhzps)
    nc2 = _round_nearest_even(r2 / dhzps)
    Nrspan = abs(nc2 - nc1) + 1
    Nrb = min(Nrb, Nrspan)
    Nrb = growNr(Nt, Nrb)
    Nr = -(-Nrspan // Nrb) * Nrb
    Nrbonus = Nr - Nrspan
    sgn = (dhzps > 0) - (dhzps < 0)
    nc1 -= _round_from_zero(sgn * Nrbonus / 2)
    nc2 += _round_to_zero(sgn * Nrbonus / 2)
    a = Fraction(nc1, Nt - 1)
    b = Fraction(nc2, Nt - 1)
    if Nr == 1:
        rs = [a]
    else:
        step = (b - a) / (Nr - 1)
        rs = [a + i * step for i in range(Nr)]
    assert len(rs) % Nrb == 0
    return [rs[i:i + Nrb] for i in range(0, len(rs), Nrb)]


# ----------------------------------------------------------------------------------------
# intfdr.jl  (bit-exact target)
# ----------------------------------------------------------------------------------------

def _julia_round(x):
    """Julia's round(x) (RoundNearest, ties to even) for a Python number."""
    if isinstance(x, Fraction):
        fl = math.floor(x)
        d = x - fl
        if d > Fraction(1, 2):
            return fl + 1
        if d < Fraction(1, 2):
            return fl
        return fl if fl % 2 == 0 else fl + 1
    return int(round(x))


def intshift_amounts(rate, Nt, rate_dtype="f64"):
    """Shift of column t: n_t = round(rate*(t)) (src/intfdr.jl:10), evaluated in the
    arithmetic of the rate's element type ("f64", "f32" or exact "rational")."""
    out = []
    for t in range(Nt):
        if rate_dtype == "f32":
            v = float(np.float32(np.float32(rate) * np.float32(t)))
        elif rate_dtype == "rational":
            v = Fraction(rate) * t
        else:
            v = float(rate) * t
        out.append(_julia_round(v))
    return out


def intshift(din, rate, rate_dtype="f64"):
    """src/intfdr.jl:7-26 -- column t circularly shifted so out[j] = in[(j + n_t) mod Nf]."""
    din = np.asarray(din)
    Nf, Nt = din.shape
    dout = np.empty_like(din)
    for t, n in enumerate(intshift_amounts(rate, Nt, rate_dtype)):
        dout[:, t] = np.roll(din[:, t], -n)
    return dout


def intfdr(spec, rates, rate_dtype="f64"):
    """src/intfdr.jl:34-61.  fdr[:, i] = sum over t (sequential, from +0.0f0, in t order,
    as Base's sum! over dims=2 accumulates) of the shifted columns, in float32."""
    spec = np.asarray(spec, dtype=np.float32)
    Nf, Nt = spec.shape
    rates = list(rates)
    fdr = np.empty((Nf, len(rates)), dtype=np.float32)
    idx = np.arange(Nf)
    for i, r in enumerate(rates):
        acc = np.zeros(Nf, dtype=np.float32)
        for t, n in enumerate(intshift_amounts(r, Nt, rate_dtype)):
            acc = acc + spec[(idx + n) % Nf, t]  # float32 + float32, rounded each step
        fdr[:, i] = acc
    return fdr


def intfdr_f64(spec, shifts):
    """FP64 truth for integer shifts: fdr[n, j] = sum_t s[(n + shifts[j][t]) mod Nf, t]."""
    spec = np.asarray(spec, dtype=np.float64)
    Nf, Nt = spec.shape
    idx = np.arange(Nf)
    out = np.zeros((Nf, len(shifts)), dtype=np.float64)
    for j, sh in enumerate(shifts):
        for t in range(Nt):
            out[:, j] += spec[(idx + int(sh[t])) % Nf, t]
    return out


# ----------------------------------------------------------------------------------------
# Float32 phase helpers (Julia cispi on a Float32 argument)
# ----------------------------------------------------------------------------------------

def cispi32(x):
    """cispi of float32 arguments, rounded to complex64.  The float32 argument is reduced
    modulo 2 exactly in float64, then cos/sin are evaluated in float64."""
    x64 = np.asarray(x, dtype=np.float32).astype(np.float64)
    r = x64 - 2.0 * np.round(x64 * 0.5)
    return (np.cos(np.pi * r) + 1j * np.sin(np.pi * r)).astype(np.complex64)


def _f32(x):
    return np.asarray(x).astype(np.float32)


# ----------------------------------------------------------------------------------------
# fftfdr.jl (FP32 mirror)
# ----------------------------------------------------------------------------------------

def phasor_arg(k, n, r, N):
    """Argument of phasor (src/fftfdr.jl:10-12): Float32(2*k*n) * r / Float32(N)."""
    kn2 = (2 * np.asarray(k, dtype=np.int64) * np.asarray(n, dtype=np.int64))
    return (_f32(kn2) * np.float32(r)) / np.float32(N)


class FFTFDRWorkspace:
    """src/fftfdr.jl:39-59: holds rfft of the spectrogram (K x Nt) and Nf."""

    def __init__(self, spec):
        spec = np.asarray(spec, dtype=np.float32)
        self.Nf, self.Nt = spec.shape
        self.dest_rfft = _fft_mod().rfft(spec, axis=0).astype(np.complex64)


def fftfdr_workspace(spec):
    return FFTFDRWorkspace(spec)


def _phasor_matrix(ws, rate):
    K = ws.dest_rfft.shape[0]
    k = np.arange(K)[:, None]
    t = np.arange(ws.Nt)[None, :]
    return cispi32(phasor_arg(k, t, np.float32(rate), ws.Nf))


def _cmul32(a, b):
    """complex64 product rounded per component as Julia's ComplexF32 `*` does."""
    a = np.asarray(a, dtype=np.complex64)
    b = np.asarray(b, dtype=np.complex64)
    ar, ai, br, bi = a.real, a.imag, b.real, b.imag
    re = (ar * br).astype(np.float32) - (ai * bi).astype(np.float32)
    im = (ar * bi).astype(np.float32) + (ai * br).astype(np.float32)
    return (re + 1j * im).astype(np.complex64)


def fdshiftsum(ws, rate):
    """src/fftfdr.jl:86-102: irfft(sum_t F .* phasor) (normalised)."""
    ph = _cmul32(ws.dest_rfft, _phasor_matrix(ws, rate))
    s = np.zeros(ph.shape[0], dtype=np.complex64)
    for t in range(ph.shape[1]):
        s = (s + ph[:, t]).astype(np.complex64)
    return _fft_mod().irfft(s, n=ws.Nf).astype(np.float32)


def fdshift(ws, rate):
    """src/fftfdr.jl:104-118: de-Dopplered spectrogram, irfft of F .* phasor per column."""
    ph = _cmul32(ws.dest_rfft, _phasor_matrix(ws, rate))
    return _fft_mod().irfft(ph, n=ws.Nf, axis=0).astype(np.float32)


def fftfdr(ws, rates):
    """src/fftfdr.jl:126-148."""
    rates = list(rates)
    out = np.empty((ws.Nf, len(rates)), dtype=np.float32)
    for j, r in enumerate(rates):
        out[:, j] = fdshiftsum(ws, r)
    return out


# ----------------------------------------------------------------------------------------
# FP64 truth: exact-phase Fourier shift sums
# ----------------------------------------------------------------------------------------

def _dyadic(x):
    """Exact (numerator, exponent) with x == num * 2**-exp for a float (or Fraction with a
    power-of-two denominator)."""
    f = Fraction(x)
    den = f.denominator
    e = den.bit_length() - 1
    if den != 1 << e:
        raise ValueError("rate is not dyadic")
    return f.numerator, e


def fdr_truth(spec, rates, workers=None):
    """FP64 Fourier-shift FDR with exact phase reduction:
    fdr[n, j] = irfft_Nf( sum_t F64[k,t] * exp(2 pi i k t r_j / Nf) )[n].

    ``rates`` are exact dyadic values (float32 values or float values converted exactly).
    The phase 2*k*t*r/Nf (half-turns) is reduced modulo 2 in integer arithmetic, so the only
    rounding is the final float64 division and the float64 cos/sin.  This is the arbiter for
    fractional rates; at integer shifts it equals the circular-shift sum.
    """
    spec = np.asarray(spec, dtype=np.float64)
    Nf, Nt = spec.shape
    F = np.fft.rfft(spec, axis=0)
    K = F.shape[0]
    k = np.arange(K, dtype=np.int64)[:, None]
    t = np.arange(Nt, dtype=np.int64)[None, :]
    kt2 = (2 * k * t)  # int64
    out = np.empty((Nf, len(rates)), dtype=np.float64)
    for j, r in enumerate(rates):
        num, e = _dyadic(r)
        # phase (half-turns) = kt2 * num / (Nf * 2**e); reduce mod 2 exactly
        mod = 2 * Nf * (1 << e)
        if abs(num) * int(kt2.max()) < (1 << 62) and mod < (1 << 62):
            rem = (kt2 * (num % mod)) % mod
        else:  # big-integer fallback (object arrays)
            rem = np.array([[(int(a) * num) % mod for a in row] for row in kt2], dtype=object)
        ph = rem.astype(np.float64) / float(Nf * (1 << e))
        ph = np.where(ph > 1.0, ph - 2.0, ph)
        S = np.sum(F * (np.cos(np.pi * ph) + 1j * np.sin(np.pi * ph)), axis=1)
        out[:, j] = np.fft.irfft(S, n=Nf)
    return out


# ----------------------------------------------------------------------------------------
# zdtfdr.jl (FP32 mirror)
# ----------------------------------------------------------------------------------------

def vlow_arg(k, l, dr, Nf):
    """Argument of vlow (src/zdtfdr.jl:140-142): Float32(-k*l^2) * dr / Float32(Nf)."""
    kl2 = -np.asarray(k, dtype=np.int64) * np.asarray(l, dtype=np.int64) ** 2
    return (_f32(kl2) * np.float32(dr)) / np.float32(Nf)


def prephase_arg(k, l, r0, dr, Nf):
    """Argument of prephase (src/zdtfdr.jl:196-198):
    Float32(k*l) * (Float32(l)*dr + 2f0*r0) / Float32(Nf)."""
    k = np.asarray(k, dtype=np.int64)
    l = np.asarray(l, dtype=np.int64)
    inner = (_f32(l) * np.float32(dr)) + np.float32(2.0) * np.float32(r0)
    return (_f32(k * l) * inner.astype(np.float32)) / np.float32(Nf)


def postphase_arg(k, l, dr, Nf):
    """Argument of postphase (src/zdtfdr.jl:268-270): Float32(k*l*l) * dr / Float32(Nf)."""
    kll = np.asarray(k, dtype=np.int64) * np.asarray(l, dtype=np.int64) ** 2
    return (_f32(kll) * np.float32(dr)) / np.float32(Nf)


def hamming(n, N):
    """src/zdtfdr.jl:303-305 (Float64)."""
    x = 2.0 * np.asarray(n, dtype=np.float64) / N
    r = x - 2.0 * np.round(x * 0.5)
    return 0.53836 + 0.46164 * np.cos(np.pi * r)


class ZDTWorkspace:
    """src/zdtfdr.jl:10-87 FP32 mirror.  Y is K x Nl complex64; Yf = Y[:, :Nt],
    Ys = Y[:, :Nr]; V = FFT_l(chirp) (K x Nl)."""

    def __init__(self, spec, r0, dr, Nr, factors=(2, 3, 5), workers=None):
        spec = np.asarray(spec, dtype=np.float32)
        self.Nf, self.Nt = spec.shape
        self.r0 = np.float32(r0)
        self.dr = np.float32(dr)
        self.Nr = int(Nr)
        self.factors = tuple(factors)
        self.Nl = calcNl(self.Nt, self.Nr, self.factors)
        self.K = self.Nf // 2 + 1
        self.workers = workers
        self.Y = np.zeros((self.K, self.Nl), dtype=np.complex64)
        self.input(spec)
        self.V = np.zeros((self.K, self.Nl), dtype=np.complex64)
        self.computeV()

    @classmethod
    def from_range(cls, spec, r0, dr, Nr, factors=(2, 3, 5), workers=None):
        return cls(spec, r0, dr, Nr, factors, workers)

    def _kw(self):
        return {"workers": self.workers} if (_sfft is not None and self.workers) else {}

    # zdtfdr.jl:173-187
    def computeV(self):
        K, Nl, Nr, Nt = self.K, self.Nl, self.Nr, self.Nt
        k = np.arange(K)[:, None]
        lo = np.arange(Nr)[None, :]
        self.V[:, :Nr] = cispi32(vlow_arg(k, lo, self.dr, self.Nf))
        if Nt > 1:
            hi = np.arange(Nl - Nt + 1, Nl)[None, :]
            self.V[:, Nl - Nt + 1:] = cispi32(vlow_arg(k, Nl - hi, self.dr, self.Nf))
        self.V = _fft_mod().fft(self.V, axis=1, **self._kw()).astype(np.complex64)

    # zdtfdr.jl:209-212
    def input(self, spec):
        spec = np.asarray(spec, dtype=np.float32)
        self.F = _fft_mod().rfft(spec, axis=0, **self._kw()).astype(np.complex64)

    # zdtfdr.jl:221-235
    def preprocess(self, r0=None):
        r0 = self.r0 if r0 is None else np.float32(r0)
        k = np.arange(self.K)[:, None]
        l = np.arange(self.Nt)[None, :]
        self.Y[:, :self.Nt] = _cmul32(self.F, cispi32(prephase_arg(k, l, r0, self.dr, self.Nf)))
        self.Y[:, self.Nt:] = 0

    # zdtfdr.jl:249-253 (ifft is the normalised ScaledPlan)
    def convolve(self):
        f = _fft_mod()
        Y = f.fft(self.Y, axis=1, **self._kw()).astype(np.complex64)
        Y = _cmul32(Y, self.V)
        self.Y = f.ifft(Y, axis=1, **self._kw()).astype(np.complex64)

    # zdtfdr.jl:297-321
    def postprocess(self, window="rect"):
        k = np.arange(self.K)[:, None]
        l = np.arange(self.Nr)[None, :]
        ph = cispi32(postphase_arg(k, l, self.dr, self.Nf))
        Ys = self.Y[:, :self.Nr]
        if window == "rect" or window is None:
            self.Y[:, :self.Nr] = _cmul32(Ys, ph)
        else:
            if window == "hamming":
                w = hamming(np.arange(self.K), self.Nf)
            elif callable(window):
                w = np.array([window(int(n), self.Nf) for n in range(self.K)], dtype=np.float64)
            else:
                raise ValueError(f"unsupported window type ({window})")
            c = ph.astype(np.complex128) * w[:, None]
            self.Y[:, :self.Nr] = (Ys.astype(np.complex128) * c).astype(np.complex64)

    # zdtfdr.jl:328-331 (normalised irfft)
    def output(self):
        return _fft_mod().irfft(self.Y[:, :self.Nr], n=self.Nf, axis=0,
                                **self._kw()).astype(np.float32)

    def zdtfdr(self, spec=None, r0=None, window="rect"):
        """zdtfdr.jl:349-421 for a single dest."""
        if spec is not None:
            self.input(spec)
        self.preprocess(r0)
        self.convolve()
        self.postprocess(window)
        return self.output()


def zdtfdr(spec, r0, dr, Nr, factors=(2, 3, 5), window="rect", workers=None):
    ws = ZDTWorkspace(spec, r0, dr, Nr, factors, workers)
    return ws.zdtfdr(window=window)


# ----------------------------------------------------------------------------------------
# fdrutils.jl
# ----------------------------------------------------------------------------------------

PAIRWISE_BLOCKSIZE = 1024  # Base.pairwise_blocksize(f, op) for sum-like reductions


def pairwise_leaves(n, blk=PAIRWISE_BLOCKSIZE):
    """Leaves of Base.mapreduce_impl(f, op, A, 1, n, blk) (Julia base/reduce.jl): a range
    [lo, hi] (1-based, inclusive) with lo == hi or hi - lo < blk is summed sequentially;
    any other range splits at mid = lo + (hi - lo) >> 1 into [lo, mid] and [mid+1, hi].
    Returned as zero-based half-open (start, stop) pairs, left to right."""
    out = []
    stack = [(1, int(n))]
    while stack:
        lo, hi = stack.pop()
        if lo == hi or hi - lo < blk:
            out.append((lo - 1, hi))
        else:
            mid = lo + ((hi - lo) >> 1)
            stack.append((mid + 1, hi))
            stack.append((lo, mid))
    return out


def pairwise_sum32(cols, f=None, blk=PAIRWISE_BLOCKSIZE):
    """Float32 sum of every column of ``cols`` (n, ncols) in the order of Julia's pairwise
    mapreduce: each leaf of ``pairwise_leaves(n)`` is summed sequentially,
    ((f(a1) + f(a2)) + f(a3)) + ..., and the leaves are combined as op(v_left, v_right) up
    the recursion.  ``f`` (float32 -> float32, elementwise on numpy arrays) defaults to
    the identity.

    The sequential leaf loop of mapreduce_impl carries Julia's ``@simd`` annotation, which
    lets LLVM reassociate it into vector lanes whose width depends on the host CPU; this
    restatement takes the loop's written (sequential) order."""
    x = np.asarray(cols, dtype=np.float32)
    if x.ndim == 1:
        x = x[:, None]
    n = x.shape[0]
    fx = x if f is None else np.asarray(f(x), dtype=np.float32)
    leaves = pairwise_leaves(n, blk)
    # sequential sums of all leaves at once: leaf l, step i adds fx[start_l + i]
    starts = np.array([a for a, _ in leaves], dtype=np.int64)
    lens = np.array([b - a for a, b in leaves], dtype=np.int64)
    acc = fx[starts].copy()                                   # (nleaves, ncols)
    for i in range(1, int(lens.max())):
        live = lens > i
        idx = starts[live] + i
        acc[live] = (acc[live] + fx[idx]).astype(np.float32)
    vals = iter(list(acc))

    def rec(lo, hi):  # same recursion as pairwise_leaves, leaves consumed left to right
        if lo == hi or hi - lo < blk:
            return next(vals)
        mid = lo + ((hi - lo) >> 1)
        a = rec(lo, mid)
        b = rec(mid + 1, hi)
        return (a + b).astype(np.float32)

    return rec(1, n)


def _std32_columns(M):
    """std(M, dims=1) in Float32 as Statistics.jl computes it (corrected): column means
    mean(M, dims=1) = pairwise sum ./ n; varm! = centralize_sumabs2! (pairwise sum of
    abs2(x - mean)) .* Float32(1 // (n-1)); then sqrt."""
    M = np.asarray(M, dtype=np.float32)
    n = M.shape[0]
    means = (pairwise_sum32(M) / np.float32(n)).astype(np.float32)
    ss = pairwise_sum32(M, f=lambda v: np.square((v - means).astype(np.float32)))
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.float32(1.0) / np.float32(n - 1)
        var = (ss * inv).astype(np.float32)
        return np.sqrt(var).astype(np.float32)


def fdrstats(fdr):
    """src/fdrutils.jl:39-50 in the reference's Float32 arithmetic: m = mean(fdr[:,1])
    (Statistics.mean: the pairwise Float32 sum of Base.mapreduce_impl divided by
    Float32(n)) of the first matrix; s = minimum over all columns (of all matrices) of
    std(fdr, dims=1) (see ``_std32_columns``), NaN if any column's std is NaN.  Returns
    (m, s) as numpy float32.  ``fdr`` may be a list of matrices."""
    mats = fdr if isinstance(fdr, (list, tuple)) else [fdr]
    c0 = np.asarray(mats[0], dtype=np.float32)[:, :1]
    m = np.float32((pairwise_sum32(c0) / np.float32(c0.shape[0]))[0])
    stds = np.concatenate([_std32_columns(M) for M in mats])
    s = np.float32(np.nan) if np.isnan(stds).any() else np.float32(stds.min())
    return m, s


def fdrstats_f64(fdr):
    """fdrstats (src/fdrutils.jl:39-50) accumulated in float64 (the statistics of the
    library's fused-moment option, which differ from the reference's Float32 pairwise
    values in the last bits)."""
    mats = fdr if isinstance(fdr, (list, tuple)) else [fdr]
    m = float(np.mean(np.asarray(mats[0][:, 0], dtype=np.float64)))
    s = min(float(np.min(np.std(np.asarray(M, dtype=np.float64), axis=0, ddof=1)))
            for M in mats)
    return m, s


def fdrnormalize(fdr, m, s):
    """src/fdrutils.jl:65-73, float32: (x - m) / s."""
    return ((np.asarray(fdr, dtype=np.float32) - np.float32(m)) / np.float32(s)).astype(np.float32)


def fdrdenormalize(snr, m, s):
    """src/fdrutils.jl:104-107: snr * s + m in Julia's promoted type.  m and s are the
    Float32 values of fdrstats.  An integer or numpy float32 ``snr`` gives Float32
    arithmetic (Int * Float32 -> Float32, each operation rounded, no fused multiply-add);
    a Python/numpy float64 ``snr`` gives Float64 arithmetic."""
    m32, s32 = np.float32(m), np.float32(s)
    if isinstance(snr, (int, np.integer, np.float32)):
        return np.float32(np.float32(np.float32(snr) * s32) + m32)
    return float(snr) * float(s32) + float(m32)


def findprotohits(fdr, threshold, snr=False):
    """src/fdrutils.jl:148-169.  Returns an (nhits, 2) int64 array of ZERO-based (i, j)
    in column-major (findall) order; for a list of matrices, j is offset by b*Nrb.  Each
    Float32 element is compared with the threshold exactly (Julia compares mixed Float32 /
    Float64 / Int values exactly).  With ``snr`` the threshold is fdrdenormalize(threshold,
    fdrstats(fdr)) in the promoted type of ``threshold`` (see ``fdrdenormalize``)."""
    mats = fdr if isinstance(fdr, (list, tuple)) else [fdr]
    thr = threshold
    if snr:
        m, s = fdrstats(mats)
        thr = fdrdenormalize(threshold, m, s)
    thr64 = float(thr)
    out = []
    Nrb = mats[0].shape[1]
    for b, M in enumerate(mats):
        j, i = np.nonzero(np.asarray(M, dtype=np.float32).T.astype(np.float64) >= thr64)
        out.append(np.stack([i, j + b * Nrb], axis=1))
    if not out:
        return np.zeros((0, 2), dtype=np.int64)
    return np.concatenate(out).astype(np.int64)


# ----------------------------------------------------------------------------------------
# Synthetic spectrograms (stand-in for the reference's Voyager-1 data)
# ----------------------------------------------------------------------------------------

def synth_spectrogram(Nf, Nt, ntones, snr_lo, snr_hi, rmax, seed):
    """Exponential(1) background plus drifting tones (power split linearly between the two
    neighbouring channels).  Returns (spec float32 (Nf, Nt), tones list of (c0, rate, amp))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.standard_normal((Nf, Nt), dtype=np.float32)
    y = rng.standard_normal((Nf, Nt), dtype=np.float32)
    spec = ((x * x + y * y) * np.float32(0.5)).astype(np.float32)
    tones = []
    for _ in range(ntones):
        c0 = rng.uniform(0, Nf)
        r = rng.uniform(-rmax, rmax)
        a = rng.uniform(snr_lo, snr_hi) if snr_hi > snr_lo else snr_lo
        tones.append((c0, r, a))
        for t in range(Nt):
            c = c0 + r * t
            c_lo = math.floor(c)
            f = c - c_lo
            spec[c_lo % Nf, t] += np.float32(a * (1.0 - f))
            spec[(c_lo + 1) % Nf, t] += np.float32(a * f)
    return spec, tones


def rel_linf(a, b):
    """max|a - b| / max|b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# ----------------------------------------------------------------------------------------
# FP64 restatement of the proposal network (gradient check of its CUDA kernels)
# ----------------------------------------------------------------------------------------

def propose_layers(nt, width=32, ksize=5, nwin=16):
    """(cin, cout, k) of the four convolution layers, in parameter order (w then b)."""
    return [(nt, width, ksize), (width, width, ksize), (width, width, ksize), (width, nwin, 1)]


def propose_unpack(params, nt, width=32, ksize=5, nwin=16):
    out, off = [], 0
    for cin, cout, k in propose_layers(nt, width, ksize, nwin):
        w = params[off:off + cout * cin * k].reshape(cout, cin, k)
        off += cout * cin * k
        b = params[off:off + cout]
        off += cout
        out.append((w, b))
    return out


def propose_loss_and_grad(params, x, labels, nt, half_weights=True):
    """Mean BCE-with-logits of the net on x (B, nt, X) and its gradient wrt params, in
    float64 (weights rounded to float16 first, as the forward pass of the kernels uses)."""
    p = np.asarray(params, np.float64)
    layers = propose_unpack(p, nt)
    if half_weights:
        layers = [(w.astype(np.float16).astype(np.float64), b) for w, b in layers]
    x = np.asarray(x, np.float64)
    B, _, X = x.shape
    acts = [x]
    for li, (w, b) in enumerate(layers):
        cout, cin, k = w.shape
        pad = k // 2
        xin = np.pad(acts[-1], ((0, 0), (0, 0), (pad, pad)))
        y = np.zeros((B, cout, X))
        for kk in range(k):
            y += np.einsum("oc,bcx->box", w[:, :, kk], xin[:, :, kk:kk + X])
        y += b[None, :, None]
        if li < 3:
            y = np.maximum(y, 0.0)
        acts.append(y)
    y4 = acts[-1]
    am = np.argmax(y4, axis=2)
    z = np.take_along_axis(y4, am[:, :, None], axis=2)[:, :, 0]
    lab = np.asarray(labels, np.float64)
    n = z.size
    loss = np.mean(np.maximum(z, 0) - z * lab + np.log1p(np.exp(-np.abs(z))))
    dz = (1.0 / (1.0 + np.exp(-z)) - lab) / n
    dy = np.zeros_like(y4)
    np.put_along_axis(dy, am[:, :, None], dz[:, :, None], axis=2)
    grads = []
    for li in range(3, -1, -1):
        w, b = layers[li]
        cout, cin, k = w.shape
        pad = k // 2
        if li < 3:
            dy = dy * (acts[li + 1] > 0)
        xin = np.pad(acts[li], ((0, 0), (0, 0), (pad, pad)))
        gw = np.zeros_like(w)
        for kk in range(k):
            gw[:, :, kk] = np.einsum("box,bcx->oc", dy, xin[:, :, kk:kk + X])
        gb = dy.sum(axis=(0, 2))
        grads.append((gw, gb))
        if li > 0:
            dpad = np.pad(dy, ((0, 0), (0, 0), (pad, pad)))
            din = np.zeros_like(acts[li])
            for kk in range(k):
                # d in[x] += w[k] * dy[x - k + pad]
                din += np.einsum("oc,box->bcx", w[:, :, kk], dpad[:, :, (k - 1 - kk):(k - 1 - kk) + X])
            dy = din
    flat = []
    for gw, gb in reversed(grads):
        flat.append(gw.ravel())
        flat.append(gb)
    return loss, np.concatenate(flat)


def _compress(v, compress):
    return np.sign(v) * np.log1p(np.abs(v)) if compress else v


def propose_features(spec, factor=256, compress=False):
    """Power input of the proposal net: (Nt, Nf/factor), (group sum - factor)/sqrt(factor),
    optionally compressed to sign(v)*log1p(|v|)."""
    s = np.asarray(spec, np.float64)
    Nf, Nt = s.shape
    g = s.reshape(Nf // factor, factor, Nt).sum(axis=1)
    return _compress(((g - factor) / math.sqrt(factor)).T, compress)


def propose_lag_features(spec, factor=256, maxlag=8, compress=False):
    """Drift evidence input: (2*maxlag+1, Nf/factor); row l+maxlag = per-bin sums over
    t < Nt-1 of (s[n,t]-1)(s[(n+l) mod Nf,t+1]-1), divided by sqrt(factor*(Nt-1))."""
    s = np.asarray(spec, np.float64) - 1.0
    Nf, Nt = s.shape
    out = np.empty((2 * maxlag + 1, Nf // factor))
    for li, l in enumerate(range(-maxlag, maxlag + 1)):
        prod = (s[:, :-1] * np.roll(s[:, 1:], -l, axis=0)).sum(axis=1)
        out[li] = prod.reshape(Nf // factor, factor).sum(axis=1)
    return _compress(out / math.sqrt(factor * (Nt - 1)), compress)


# ----------------------------------------------------------------------------------------
# Proto-hits -> hits (connected components; the step after findprotohits)
# ----------------------------------------------------------------------------------------

def cluster_protohits(hits, Nf, di=1, dj=1, fdr=None):
    """Union-find restatement of the device clustering: proto-hits (zero-based (i, j), in
    column-major order) touch when |Δi| <= di and |Δj| <= dj (no wrap).  Returns
    (labels, clusters): clusters numbered by their first proto-hit, each a dict with
    count, i_min, i_max, j_min, j_max, first, peak_i, peak_j, peak_value (largest FDR value,
    earliest proto-hit on ties; the first proto-hit and NaN without an FDR)."""
    hits = np.asarray(hits, dtype=np.int64).reshape(-1, 2)
    n = len(hits)
    index = {(int(i), int(j)): h for h, (i, j) in enumerate(hits)}
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for h, (i, j) in enumerate(hits):
        for dc in range(-dj, dj + 1):
            for dr in range(-di, di + 1):
                if not (0 <= int(i) + dr < Nf):
                    continue
                g = index.get((int(i) + dr, int(j) + dc))
                if g is None:
                    continue
                a, b = find(h), find(g)
                if a != b:
                    parent[max(a, b)] = min(a, b)
    roots = [find(h) for h in range(n)]
    order = sorted(set(roots))
    cid = {r: c for c, r in enumerate(order)}
    labels = np.array([cid[r] for r in roots], dtype=np.int64)
    mats = None
    if fdr is not None:
        mats = fdr if isinstance(fdr, (list, tuple)) else [fdr]
    members_of = {r: [] for r in order}
    for h, r in enumerate(roots):
        members_of[r].append(h)
    clusters = []
    for r in order:
        members = members_of[r]
        ii, jj = hits[members, 0], hits[members, 1]
        if mats is not None:
            Nrb = mats[0].shape[1]
            vals = [np.float32(mats[int(j) // Nrb][int(i), int(j) % Nrb]) for i, j in zip(ii, jj)]
            best = max(range(len(members)), key=lambda m: (vals[m], -members[m]))
            pv = float(vals[best])
        else:
            best, pv = 0, float("nan")
        clusters.append({"count": len(members), "i_min": int(ii.min()), "i_max": int(ii.max()),
                         "j_min": int(jj.min()), "j_max": int(jj.max()), "first": int(r),
                         "peak_i": int(ii[best]), "peak_j": int(jj[best]), "peak_value": pv})
    return labels, clusters


# ----------------------------------------------------------------------------------------
# Taylor tree (the faster integer FDR that the reference's README.md:88-92 mentions)
# ----------------------------------------------------------------------------------------

def taylor_tree(spec, dmin, dmax):
    """Float32 restatement of the Taylor-tree FDR with the device's addition order: stage by
    stage, row (block*2L + d) = row (2*block*L + d//2) + row ((2*block+1)*L + d//2) shifted by
    ceil(d/2) channels (circularly; towards lower channels for the negative tree).  Returns
    (Nf, dmax-dmin+1) float32, column d - dmin."""
    s = np.asarray(spec, dtype=np.float32)
    Nf, Nt = s.shape
    assert Nt & (Nt - 1) == 0
    out = np.empty((Nf, dmax - dmin + 1), dtype=np.float32)
    for sgn in (+1, -1):
        A = s.T.copy()  # rows = steps
        L = 1
        while L < Nt:
            B = np.empty_like(A)
            for blk in range(Nt // (2 * L)):
                for d in range(2 * L):
                    top = A[2 * blk * L + d // 2]
                    bot = np.roll(A[(2 * blk + 1) * L + d // 2], -sgn * ((d + 1) // 2))
                    B[blk * 2 * L + d] = top + bot
            A = B
            L *= 2
        for d in range(dmin, dmax + 1):
            if (d >= 0) == (sgn > 0):
                out[:, d - dmin] = A[abs(d)]
    return out


# ----------------------------------------------------------------------------------------
# Threaded CPU restatement of zdtfdr! for timing the reference's CPU path
# ----------------------------------------------------------------------------------------

class ThreadedZDT:
    """zdtfdr!(dest, ws, spectrogram) restated for speed on the host cores, for timing the
    reference's CPU path (the reference itself is Julia + FFTW, which is not installed).
    Same stage order as src/zdtfdr.jl:349-362 -- input! (rfft), preprocess! (prephase
    multiply and zero fill of Y), convolve! (FFT over l, x V, normalised inverse FFT),
    postprocess! (postphase multiply), output! (normalised irfft) -- with the chirp factors
    computed per call from the reference's Float32 phase arguments (prephase_arg,
    postphase_arg), as the reference's broadcasts do.  Arithmetic is complex64 (numpy's
    complex multiply, not the per-component rounding of ``_cmul32``); FFTs are scipy
    pocketfft with ``workers`` threads; the elementwise stages run on row blocks in a pool
    of ``workers`` threads.  V is built once, as ZDTWorkspace does."""

    def __init__(self, spec, r0, dr, Nr, workers=None, factors=(2, 3, 5)):
        import concurrent.futures as cf
        import os
        spec = np.asarray(spec, dtype=np.float32)
        self.Nf, self.Nt = spec.shape
        self.r0, self.dr, self.Nr = np.float32(r0), np.float32(dr), int(Nr)
        self.Nl = calcNl(self.Nt, self.Nr, factors)
        self.K = self.Nf // 2 + 1
        self.workers = int(workers or os.cpu_count() or 1)
        self.pool = cf.ThreadPoolExecutor(self.workers)
        self.V = ZDTWorkspace(spec, r0, dr, Nr, factors, workers=self.workers).V  # (K, Nl)
        self.Y = np.empty((self.K, self.Nl), dtype=np.complex64)
        self.F = None
        bl = max(1, -(-self.K // (4 * self.workers)))
        self.blocks = [(a, min(self.K, a + bl)) for a in range(0, self.K, bl)]

    def _par(self, fn):
        list(self.pool.map(lambda ab: fn(*ab), self.blocks))

    def zdtfdr(self, spec):
        f = _fft_mod()
        w = {"workers": self.workers} if _sfft is not None else {}
        spec = np.asarray(spec, dtype=np.float32)
        self.F = f.rfft(spec, axis=0, **w).astype(np.complex64, copy=False)     # input!
        Nt, Nr, Nf = self.Nt, self.Nr, self.Nf
        lt = np.arange(Nt)[None, :]
        lr = np.arange(Nr)[None, :]

        def pre(a, b):                                                          # preprocess!
            k = np.arange(a, b)[:, None]
            self.Y[a:b, :Nt] = self.F[a:b] * cispi32(prephase_arg(k, lt, self.r0, self.dr, Nf))
            self.Y[a:b, Nt:] = 0
        self._par(pre)
        Y = f.fft(self.Y, axis=1, **w)                                          # convolve!
        self._par(lambda a, b: np.multiply(Y[a:b], self.V[a:b], out=Y[a:b]))
        Y = f.ifft(Y, axis=1, overwrite_x=True, **w)

        def post(a, b):                                                         # postprocess!
            k = np.arange(a, b)[:, None]
            Y[a:b, :Nr] *= cispi32(postphase_arg(k, lr, self.dr, Nf))
        self._par(post)
        return f.irfft(Y[:, :Nr], n=Nf, axis=0, **w).astype(np.float32, copy=False)  # output!


# ----------------------------------------------------------------------------------------
# Bitshuffle/LZ4 chunks of rawspec's HDF5 products (test/heavytests.jl:11-14 reads them
# through HDF5.jl + H5Zbitshuffle.jl; the filter is a third-party dependency, restated here
# from the published bitshuffle and LZ4 block formats)
# ----------------------------------------------------------------------------------------

def lz4_block_decode(src):
    """LZ4 block format: sequences of a token (high nibble literal count, low nibble match
    length - 4, each 15 extended by following bytes until one is < 255), the literals, then
    (except for the last sequence) a 2-byte little-endian offset back into the output and a
    copy of the match length, byte by byte so that overlapping copies repeat."""
    src = bytes(src)
    out = bytearray()
    ip = 0
    while ip < len(src):
        tok = src[ip]
        ip += 1
        lit = tok >> 4
        if lit == 15:
            while True:
                b = src[ip]
                ip += 1
                lit += b
                if b != 255:
                    break
        out += src[ip:ip + lit]
        ip += lit
        if ip >= len(src):
            break
        off = src[ip] | (src[ip + 1] << 8)
        ip += 2
        if off == 0 or off > len(out):
            raise ValueError("lz4: bad offset")
        ml = tok & 15
        if ml == 15:
            while True:
                b = src[ip]
                ip += 1
                ml += b
                if b != 255:
                    break
        ml += 4
        for _ in range(ml):
            out.append(out[-off])
    return bytes(out)


def bitshuffle_block(data, elem_size):
    """Bit transpose of one block of n elements (n a multiple of 8): output bit-row
    8*j + k (byte j of the little-endian element, bit k, least significant first) holds bit
    k of byte j of every element, element e at bit (e mod 8) of byte e // 8 of the row."""
    a = np.frombuffer(bytes(data), dtype=np.uint8).reshape(-1, elem_size)   # (n, es)
    bits = np.unpackbits(a, axis=1, bitorder="little").reshape(-1, elem_size, 8)  # (n, j, k)
    rows = bits.transpose(1, 2, 0).reshape(elem_size * 8, -1)               # (8j+k, n)
    return np.packbits(rows, axis=1, bitorder="little").tobytes()


def bitunshuffle_block(data, elem_size):
    """Inverse of ``bitshuffle_block``."""
    rows = np.frombuffer(bytes(data), dtype=np.uint8).reshape(elem_size * 8, -1)
    bits = np.unpackbits(rows, axis=1, bitorder="little")                   # (8j+k, n)
    n = bits.shape[1]
    b = bits.reshape(elem_size, 8, n).transpose(2, 0, 1)                    # (n, j, k)
    return np.packbits(b, axis=2, bitorder="little").reshape(n * elem_size).tobytes()


def bitshuffle_lz4_decode_chunk(chunk, elem_size):
    """A bitshuffle+LZ4 chunk to its elements' bytes: 8-byte big-endian uncompressed size,
    4-byte big-endian block size in bytes, then per block (the last one holding the
    remaining whole groups of 8 elements) a 4-byte big-endian compressed size and an LZ4
    block of bit-transposed elements, then the remaining (elements mod 8) elements raw."""
    chunk = bytes(chunk)
    total = int.from_bytes(chunk[0:8], "big")
    bbytes = int.from_bytes(chunk[8:12], "big")
    nelem = total // elem_size
    bel = bbytes // elem_size
    whole = nelem - nelem % 8
    ip, out = 12, bytearray()
    e0 = 0
    while e0 < whole:
        ne = min(bel, whole - e0)
        csz = int.from_bytes(chunk[ip:ip + 4], "big")
        ip += 4
        blk = lz4_block_decode(chunk[ip:ip + csz])
        if len(blk) != ne * elem_size:
            raise ValueError("bitshuffle: block size mismatch")
        out += bitunshuffle_block(blk, elem_size)
        ip += csz
        e0 += ne
    out += chunk[ip:ip + (nelem - whole) * elem_size]
    return bytes(out)
