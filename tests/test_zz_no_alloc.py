"""GPU test of fdr_stats_noalloc, the statistics entry point that allocates no device
memory, for callers that may not allocate while running: real-time pipelines (an allocation
can stall or fail mid-run) and hosts whose device memory belongs to their own pool.  It is
called through the C ABI and compared, bit for bit, with fdr_stats (the allocating entry
point) and with the oracle's Float32 restatement of fdrstats, on calls in a row: different
matrices (the shared scratch array keeps the previous call's contents), the same matrix
twice, and the column-count limit.  Collected last so that a stop-at-first-failure run has
run every other test first."""
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


def _oracle_stats(oracle, a):
    m, s = oracle.fdrstats(a)
    return float(m), float(s)


def test_stats_noalloc_matches_fdr_stats(fdr, oracle):
    lib = fdr._lib.lib()
    torch.cuda.init()
    mats = []
    for seed, (Nf, Nr) in [(1, (65536, 33)), (2, (4096, 129)), (3, (3000, 7))]:
        spec, _ = oracle.synth_spectrogram(Nf, 16, 3, 20, 20, 4, seed=seed)
        mats.append(oracle.intfdr(spec, [-4.0 + 0.25 * j for j in range(Nr)]))
    for a in mats:  # calls in a row on different data
        g = fdr.as_device_f32(a)
        ref = _oracle_stats(oracle, a)
        assert _stats_noalloc(lib, g) == ref
        assert _stats_alloc(lib, g) == ref
    g = fdr.as_device_f32(mats[0])  # the same matrix twice in a row
    first = _stats_noalloc(lib, g)
    assert _stats_noalloc(lib, g) == first == _oracle_stats(oracle, mats[0])


def test_stats_noalloc_at_column_limit(fdr, oracle):
    """Nr = FDR_STATS_NOALLOC_MAX_COLUMNS (8192), where the partial sums fill the array."""
    lib = fdr._lib.lib()
    rng = np.random.default_rng(11)
    a = (rng.exponential(1.0, (2048, 8192)) * 3).astype(np.float32)
    a[:, 4097] *= np.float32(0.5)  # the column of least std is not the first
    g = fdr.as_device_f32(a)
    ref = _oracle_stats(oracle, a)
    assert _stats_noalloc(lib, g) == ref
    assert _stats_alloc(lib, g) == ref


def test_stats_noalloc_rejects_too_many_columns(fdr):
    lib = fdr._lib.lib()
    g = torch.zeros((8193, 2), dtype=torch.float32, device="cuda")  # Nf=2, Nr=8193 columns
    m, s = C.c_double(), C.c_double()
    st = lib.fdr_stats_noalloc(C.c_void_p(g.data_ptr()), 2, 8193, C.byref(m), C.byref(s), None)
    assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT
    assert b"8192" in lib.fdr_last_error_string()
