"""Mixed-precision ZDT (FDR_ZDT_MIXED_PRECISION): the output pass's DFTs as split-bfloat16
tensor-core contractions.  Tolerances (relative L-infinity of the FDR's peak): 1e-4 against
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
    """Shapes without the P = 1024 split run the float32 kernels unchanged."""
    spec, d, ws32, wsm = _setup(fdr, oracle, 1 << 16, 16, 33, seed=9)
    assert np.array_equal(fdr.zdtfdr(ws32).cpu().numpy(), fdr.zdtfdr(wsm).cpu().numpy())
