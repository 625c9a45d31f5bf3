"""Mixed-precision ZDT (FDR_ZDT_MIXED_PRECISION): the output pass's DFTs as split-bfloat16
tensor-core contractions (tcgen05 with tensor-memory accumulators for P = 2048, mma.sync for
P = 1024).  Tolerances (relative L-infinity of the FDR's peak): 1e-4 against
FP64 (the accuracy bound of the FDR; measured ~2e-6) and 2e-5 against the FP32 plain form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(fdr, oracle, Nf, Nt, Nr, seed):
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 20, 8.0, 50.0, 4.0, seed=seed)
    d = fdr.as_device_f32(spec)
    return spec, d, fdr.ZDTWorkspace(d, -4.0, 1 / 16, Nr), \
        fdr.ZDTWorkspace(d, -4.0, 1 / 16, Nr, mixed_precision=True)


def test_mixed_error_bounds(fdr, oracle):
    Nf, Nt, Nr = 1 << 20, 16, 129
    spec, d, ws32, wsm = _setup(fdr, oracle, Nf, Nt, Nr, seed=3)
    a = fdr.zdtfdr(ws32).cpu().numpy()
    b = fdr.zdtfdr(wsm).cpu().numpy()
    fdr.fdrsynchronize()
    e32 = oracle.rel_linf(b, a)
    assert e32 < 2e-5, e32
    assert oracle.rel_l2(b, a) < 2e-5
    cols = [0, 37, 128]
    truth = oracle.fdr_truth(spec, [-4.0 + j / 16 for j in cols])
    e64 = oracle.rel_linf(b[:, cols], truth)
    print(f"mixed: rel Linf vs FP32 {e32:.2e}, vs FP64 {e64:.2e}")
    assert e64 < 1e-4, e64
    assert not np.array_equal(a, b)  # the tensor-core path ran


def test_mixed_protohits_and_subsets(fdr, oracle):
    Nf, Nt, Nr = 1 << 20, 16, 65
    spec, d, ws32, wsm = _setup(fdr, oracle, Nf, Nt, Nr, seed=8)
    h32 = fdr.zdtfdr_protohits_(fdr.fortran_empty(Nf, Nr), ws32, d, threshold=10.0)
    hm = fdr.zdtfdr_protohits_(fdr.fortran_empty(Nf, Nr), wsm, d, threshold=10.0)
    a, b = set(map(tuple, h32.tolist())), set(map(tuple, hm.tolist()))
    assert len(a) > 0 and len(a & b) >= 0.999 * len(a) and len(a & b) >= 0.999 * len(b)
    full = fdr.zdtfdr(wsm).cpu().numpy()
    sub = fdr.fortran_empty(Nf, 16)
    fdr.zdtfdr_blocks_(sub, wsm, d, [6, 1])
    assert np.array_equal(sub.cpu().numpy(), full[:, list(range(48, 56)) + list(range(8, 16))])


def test_mixed_flag_other_shapes_use_fp32(fdr, oracle):
    """Shapes whose split has neither P = 1024 nor P = 2048 run the float32 kernels unchanged."""
    spec, d, ws32, wsm = _setup(fdr, oracle, 1 << 16, 16, 33, seed=9)
    assert np.array_equal(fdr.zdtfdr(ws32).cpu().numpy(), fdr.zdtfdr(wsm).cpu().numpy())


@pytest.mark.parametrize("Nf,Nt,Nr,split", [
    (1 << 21, 16, 33, (2048, 1024)),  # tcgen05 output pass, 1024 residues
    (1 << 20, 12, 17, (2048, 512)),   # tcgen05, odd Nr: the last rate pair holds one rate
    (1 << 19, 16, 33, (1024, 512)),   # mma.sync output pass (P = 1024)
])
def test_mixed_output_passes(fdr, oracle, Nf, Nt, Nr, split):
    """Both tensor-core output passes against the float32 form (2e-5) and FP64 (1e-4) on
    sampled columns; the mixed workspace takes the plain form's four-step split."""
    assert fdr.fused_split(Nf, Nt, Nr, mixed_precision=True) == split
    spec, d, ws32, wsm = _setup(fdr, oracle, Nf, Nt, Nr, seed=Nf % 97 + Nr)
    a = fdr.zdtfdr(ws32).cpu().numpy()
    b = fdr.zdtfdr(wsm).cpu().numpy()
    fdr.fdrsynchronize()
    assert not np.array_equal(a, b)  # a tensor-core pass ran
    assert oracle.rel_linf(b, a) < 2e-5
    cols = [0, Nr // 2, Nr - 1]
    truth = oracle.fdr_truth(spec, [-4.0 + j / 16 for j in cols])
    assert oracle.rel_linf(b[:, cols], truth) < 1e-4


def test_mixed_snr_search_and_fast_stats(fdr, oracle):
    """The snr proto-hit search on a mixed-precision FDR equals findprotohits on that FDR,
    with the statistics of the pairwise pass and with the float64 moments that the tcgen05
    output pass accumulates (fast_stats)."""
    Nf, Nt, Nr = 1 << 20, 16, 65
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 20, 8.0, 50.0, 4.0, seed=77)
    d = fdr.as_device_f32(spec)
    ws = fdr.ZDTWorkspace(d, -4.0, 1 / 16, Nr, mixed_precision=True)
    dest = fdr.fortran_empty(Nf, Nr)
    hits = fdr.zdtfdr_protohits_(dest, ws, d, threshold=6, snr=True)
    F = dest.cpu().numpy()
    assert len(hits) > 0
    assert np.array_equal(hits, oracle.findprotohits(F, 6, snr=True))
    wsf = fdr.ZDTWorkspace(d, -4.0, 1 / 16, Nr, mixed_precision=True, fast_stats=True)
    dest2 = fdr.fortran_empty(Nf, Nr)
    hits2, thr = fdr.zdtfdr_protohits_(dest2, wsf, d, threshold=6.0, snr=True, return_threshold=True)
    F2 = dest2.cpu().numpy()
    assert np.array_equal(F, F2)
    m64, s64 = oracle.fdrstats_f64(F2)
    ref_thr = 6.0 * float(np.float32(s64)) + float(np.float32(m64))
    assert abs(thr - ref_thr) <= 1e-6 * ref_thr
    assert np.array_equal(hits2, oracle.findprotohits(F2, thr))
