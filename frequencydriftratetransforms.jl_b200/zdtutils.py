"""zdtutils.jl host helpers (calcNl, growNr, estimate_memory, driftrates)."""
from __future__ import annotations

import numpy as np

from . import _lib


def _factors(factors):
    return _lib.i64_array([int(f) for f in factors])


def calcNl(Nt, Nr, factors=(2, 3, 5)):
    """zdtutils.jl:7-9 -- smallest 'factors'-smooth integer >= Nt + Nr - 1."""
    arr, n = _factors(factors)
    v = _lib.lib().fdr_calc_nl(int(Nt), int(Nr), arr, n)
    if v < 0:
        raise ValueError("calcNl: invalid arguments")
    return int(v)


def growNr(Nt, Nr, factors=(2, 3, 5)):
    """zdtutils.jl:17-19."""
    arr, n = _factors(factors)
    v = _lib.lib().fdr_grow_nr(int(Nt), int(Nr), arr, n)
    if v < 0:
        raise ValueError("growNr: invalid arguments")
    return int(v)


def estimate_memory(Nf, Nt, Nr, Ni=1, No=1, factors=(2, 3, 5)):
    """zdtutils.jl:35-53 (the reference's formula, bytes)."""
    arr, n = _factors(factors)
    v = _lib.lib().fdr_estimate_memory(int(Nf), int(Nt), int(Nr), int(Ni), int(No), arr, n)
    if v < 0:
        raise ValueError("estimate_memory: invalid arguments")
    return int(v)


def driftrates(ws, r0=None):
    """zdtutils.jl:62-64 -- the workspace's normalised drift rates as float32 values
    (element j is the float32 rounding of r0 + j*dr)."""
    r0 = np.float32(ws.r0 if r0 is None else r0)
    dr = np.float32(ws.dr)
    return (float(r0) + np.arange(ws.Nr, dtype=np.float64) * float(dr)).astype(np.float32)
