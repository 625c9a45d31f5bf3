"""GPU tests of fdrstats / fdrnormalize! / findprotohits (fdrutils.jl)."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _fdr(oracle, Nf=65536, Nr=33, seed=1):
    spec, _ = oracle.synth_spectrogram(Nf, 16, 3, 20, 20, 4, seed=seed)
    return oracle.intfdr(spec, [-4.0 + 0.25 * j for j in range(Nr)])


def test_stats(fdr, oracle):
    """fdrstats in the reference's Float32 pairwise order: bit-exact with the oracle."""
    a = _fdr(oracle)
    m, s = fdr.fdrstats(fdr.as_device_f32(a))
    mr, sr = oracle.fdrstats(a)
    assert (m, s) == (mr, sr)
    b = _fdr(oracle, seed=2)
    m2, s2 = fdr.fdrstats([fdr.as_device_f32(a), fdr.as_device_f32(b)])
    assert (m2, s2) == oracle.fdrstats([a, b])


@pytest.mark.parametrize("Nf,Nr", [(1, 3), (2, 2), (15, 4), (16, 3), (17, 5), (1024, 3), (1025, 2),
                                   (3000, 7), (8195, 3), (12289, 2), (1 << 16, 1), (100003, 2)])
def test_stats_ragged_lengths_bit_exact(fdr, oracle, Nf, Nr):
    """Column lengths whose pairwise recursion has leaves at two depths, single-element
    columns (std NaN: 0 * Float32(1//0)) and unaligned leaves."""
    rng = np.random.default_rng(Nf * 7 + Nr)
    a = (rng.exponential(1.0, (Nf, Nr)) * 16).astype(np.float32)
    m, s = fdr.fdrstats(fdr.as_device_f32(a))
    mr, sr = oracle.fdrstats(a)
    assert m == mr
    assert (np.isnan(s) and np.isnan(sr)) or s == sr


def test_normalize_bit_exact(fdr, oracle):
    a = _fdr(oracle)
    m, s = np.float32(16.25), np.float32(3.75)
    g = fdr.as_device_f32(a.copy())
    fdr.fdrnormalize_(g, m, s)
    ref = oracle.fdrnormalize(a, m, s)
    assert np.array_equal(g.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    assert fdr.fdrnormalize(20.0, 16.0, 2.0) == 2.0
    assert fdr.fdrdenormalize(10, 16.0, 2.0) == 36.0


@pytest.mark.parametrize("thr", [30.0, 45.5, 1e9])
def test_findprotohits_exact(fdr, oracle, thr):
    a = _fdr(oracle)
    hits = fdr.findprotohits(fdr.as_device_f32(a), thr)
    ref = oracle.findprotohits(a, thr)
    assert np.array_equal(hits, ref)


def test_findprotohits_snr_and_batches(fdr, oracle):
    a, b = _fdr(oracle, seed=3), _fdr(oracle, seed=4)
    ga, gb = fdr.as_device_f32(a), fdr.as_device_f32(b)
    mr, sr = oracle.fdrstats([a, b])
    for snr in (8.0, 8):  # Float64 and Int snr (Float32 arithmetic)
        hits, thr = fdr.findprotohits([ga, gb], snr, snr=True, return_threshold=True)
        thr_ref = oracle.fdrdenormalize(snr, mr, sr)
        assert thr == float(thr_ref)
        assert np.array_equal(hits, oracle.findprotohits([a, b], snr, snr=True))
        assert hits[:, 1].max() >= a.shape[1]  # offsets of the second matrix


def test_findprotohits_capacity(fdr, oracle):
    a = _fdr(oracle, Nf=4096, Nr=5)
    g = fdr.as_device_f32(a)
    lib = fdr._lib.lib()
    buf = torch.empty((4, 2), dtype=torch.int64, device="cuda")
    cnt = C.c_int64()
    ptrs = (C.c_void_p * 1)(g.data_ptr())
    st = lib.fdr_findprotohits(ptrs, 1, 4096, 5, 0.0, 0, C.c_void_p(buf.data_ptr()), 4,
                               C.byref(cnt), None, None)
    assert st == fdr._lib.FDR_ERR_CAPACITY and cnt.value == 4096 * 5
    ref = oracle.findprotohits(a, 0.0)
    assert np.array_equal(buf.cpu().numpy(), ref[:4])
    # the Python wrapper grows its buffer and retries
    assert len(fdr.findprotohits(g, 0.0, capacity=16)) == 4096 * 5


@pytest.mark.parametrize("Nf,Nr", [(1, 3), (2, 2), (15, 4), (17, 5), (1024, 3), (1025, 2),
                                   (3000, 7), (8195, 3), (12289, 2), (1 << 16, 2), (100003, 2)])
def test_findprotohits_snr_ragged_lengths(fdr, oracle, Nf, Nr):
    """The snr search reads again only the pairwise leaves whose maximum reaches the
    threshold: hit lists equal the oracle's full scan for ragged column lengths, for sparse
    (snr 2), dense (snr 0.25) and almost-everything (snr -1) thresholds, in both snr types."""
    rng = np.random.default_rng(Nf * 5 + Nr)
    a = (rng.exponential(1.0, (Nf, Nr)) * 16).astype(np.float32)
    g = fdr.as_device_f32(a)
    for snr in (2.0, 0.25, -1, 2):
        hits, thr = fdr.findprotohits(g, snr, snr=True, return_threshold=True)
        ref = oracle.findprotohits(a, snr, snr=True)
        assert np.array_equal(hits, ref), (snr, len(hits), len(ref))
        if Nf == 1:
            assert np.isnan(thr) and len(hits) == 0  # std of one element is NaN


def test_findprotohits_snr_nan_column(fdr, oracle):
    """A NaN anywhere makes its column's std NaN, so the threshold is NaN and nothing is a
    hit; a NaN inside a leaf never becomes that leaf's maximum."""
    a = _fdr(oracle, Nf=8192, Nr=4)
    a[5000, 2] = np.nan
    g = fdr.as_device_f32(a)
    hits, thr = fdr.findprotohits(g, 1.0, snr=True, return_threshold=True)
    assert np.isnan(thr) and len(hits) == 0
    assert len(oracle.findprotohits(a, 1.0, snr=True)) == 0


def test_findprotohits_snr_capacity(fdr, oracle):
    """With snr and too small a buffer: FDR_ERR_CAPACITY, the true count and threshold, and
    the first `capacity` hits in order."""
    a = _fdr(oracle, Nf=3000, Nr=5)
    g = fdr.as_device_f32(a)
    lib = fdr._lib.lib()
    ref = oracle.findprotohits(a, 0.5, snr=True)
    assert len(ref) > 40
    buf = torch.empty((40, 2), dtype=torch.int64, device="cuda")
    cnt, thr = C.c_int64(), C.c_double()
    ptrs = (C.c_void_p * 1)(g.data_ptr())
    st = lib.fdr_findprotohits(ptrs, 1, 3000, 5, 0.5, fdr._lib.FDR_SNR_F64,
                               C.c_void_p(buf.data_ptr()), 40, C.byref(cnt), C.byref(thr), None)
    assert st == fdr._lib.FDR_ERR_CAPACITY and cnt.value == len(ref)
    mr, sr = oracle.fdrstats(a)
    assert thr.value == float(oracle.fdrdenormalize(0.5, mr, sr))
    assert np.array_equal(buf.cpu().numpy(), ref[:40])


def test_hit_buffer_memory_kinds(fdr, oracle):
    """The hit buffer may be device memory or pinned (mapped) host memory, which the kernels
    write directly; pageable host memory is rejected before any kernel runs."""
    a = _fdr(oracle, Nf=4096, Nr=5)
    g = fdr.as_device_f32(a)
    lib = fdr._lib.lib()
    ref = oracle.findprotohits(a, 40.0)
    ptrs = (C.c_void_p * 1)(g.data_ptr())
    for mode, thr in ((0, 40.0), (fdr._lib.FDR_SNR_F64, 2.0)):
        want = ref if mode == 0 else oracle.findprotohits(a, thr, snr=True)
        pinned = torch.zeros((len(want) + 3, 2), dtype=torch.int64, pin_memory=True)
        cnt = C.c_int64()
        st = lib.fdr_findprotohits(ptrs, 1, 4096, 5, thr, mode, C.c_void_p(pinned.data_ptr()),
                                   len(want) + 3, C.byref(cnt), None, None)
        assert st == 0 and cnt.value == len(want)
        assert np.array_equal(pinned[: cnt.value].numpy(), want)
        pageable = np.zeros((len(want) + 3, 2), dtype=np.int64)
        st = lib.fdr_findprotohits(ptrs, 1, 4096, 5, thr, mode,
                                   C.c_void_p(pageable.ctypes.data), len(want) + 3,
                                   C.byref(cnt), None, None)
        assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT
        assert not pageable.any()
