"""GPU test of fdr_stats_noalloc, the statistics entry point that allocates no device
memory (for callers that may not allocate while running: real-time pipelines, hosts whose
device memory belongs to their own pool).  It is called through the C ABI and compared
with fdr_stats, the allocating entry point, on two calls in a row (the shared scratch array
keeps the previous call's contents, so the second call checks that it is cleared).
Collected last so that a stop-at-first-failure run has run every other test first."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _stats_alloc(lib, g):
    m, s = C.c_double(), C.c_double()
    ptrs = (C.c_void_p * 1)(g.data_ptr())
    assert lib.fdr_stats(ptrs, 1, g.shape[0], g.shape[1], C.byref(m), C.byref(s), None) == 0
    return m.value, s.value


def _stats_noalloc(lib, g):
    m, s = C.c_double(), C.c_double()
    st = lib.fdr_stats_noalloc(C.c_void_p(g.data_ptr()), g.shape[0], g.shape[1], C.byref(m),
                               C.byref(s), None)
    assert st == 0, lib.fdr_last_error_string()
    return m.value, s.value


def test_stats_noalloc_matches_fdr_stats(fdr, oracle):
    lib = fdr._lib.lib()
    torch.cuda.init()
    mats = []
    for seed, (Nf, Nr) in [(1, (65536, 33)), (2, (4096, 129))]:
        spec, _ = oracle.synth_spectrogram(Nf, 16, 3, 20, 20, 4, seed=seed)
        mats.append(fdr.as_device_f32(oracle.intfdr(spec, [-4.0 + 0.25 * j for j in range(Nr)])))
    for g in mats:  # two calls in a row on different data
        m0, s0 = _stats_alloc(lib, g)
        m1, s1 = _stats_noalloc(lib, g)
        assert abs(m1 - m0) <= 1e-9 * abs(m0)
        assert abs(s1 - s0) <= 1e-9 * abs(s0)


def test_stats_noalloc_rejects_too_many_columns(fdr):
    lib = fdr._lib.lib()
    g = torch.zeros((8193, 2), dtype=torch.float32, device="cuda")  # Nf=2, Nr=8193 columns
    m, s = C.c_double(), C.c_double()
    st = lib.fdr_stats_noalloc(C.c_void_p(g.data_ptr()), 2, 8193, C.byref(m), C.byref(s), None)
    assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT
    assert b"8192" in lib.fdr_last_error_string()
