"""GPU tests of the Fourier-shift FDR (fftfdr.jl) against the oracle.

Tolerance: relative L-infinity 2e-5 vs the FP32 mirror, 1e-5 vs FP64 at these sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_known_answers(fdr, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    ws = fdr.fftfdr_workspace(d)
    np.testing.assert_allclose(fdr.fdshift(ws, 1).cpu().numpy(),
                               np.array(golden["intshift_expected"]), atol=2e-6)
    np.testing.assert_allclose(fdr.fftfdr(ws, golden["rates"]).cpu().numpy(),
                               np.array(golden["fdr_expected"]), atol=2e-6)


@pytest.mark.parametrize("Nf,Nt", [(4096, 16), (1000, 7), (65536, 16), (2 ** 20, 16)])
def test_fftfdr_vs_oracle(fdr, oracle, Nf, Nt):
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 20, 20, 4, seed=Nf)
    rates = [-4.0 + 0.25 * j for j in range(33)]
    if Nf >= 2 ** 20:
        rates = rates[::8]
    ws = fdr.fftfdr_workspace(spec)
    out = fdr.fftfdr(ws, rates).cpu().numpy()
    mws = oracle.fftfdr_workspace(spec)
    assert oracle.rel_linf(out, oracle.fftfdr(mws, rates)) < 2e-5
    assert oracle.rel_linf(out, oracle.fdr_truth(spec, rates)) < 1e-4
    # a lone column is transformed with a zero partner, a column of fftfdr with its
    # neighbour (two-for-one real FFT): equal up to float32 rounding
    col = fdr.fdshiftsum(ws, rates[1]).cpu().numpy()
    assert oracle.rel_linf(col, out[:, 1]) < 1e-6


def test_fdshift_vs_oracle(fdr, oracle):
    spec, _ = oracle.synth_spectrogram(2048, 16, 2, 20, 20, 4, seed=8)
    ws = fdr.fftfdr_workspace(spec)
    mws = oracle.fftfdr_workspace(spec)
    for r in [-2.43, 0.0, 1.5]:
        out = fdr.fdshift(ws, r).cpu().numpy()
        assert oracle.rel_linf(out, oracle.fdshift(mws, r)) < 2e-5


def test_workspace_update_and_size_check(fdr, oracle):
    s1, _ = oracle.synth_spectrogram(1024, 8, 1, 20, 20, 2, seed=1)
    s2, _ = oracle.synth_spectrogram(1024, 8, 1, 20, 20, 2, seed=2)
    ws = fdr.fftfdr_workspace(s1)
    fdr.fftfdr_workspace_(ws, s2)
    out = fdr.fftfdr(ws, [0.5]).cpu().numpy()
    ref = oracle.fftfdr(oracle.fftfdr_workspace(s2), [0.5])
    assert oracle.rel_linf(out, ref) < 2e-5
    with pytest.raises(fdr.FDRError):
        fdr.fftfdr_workspace_(ws, np.zeros((1024, 9), dtype=np.float32))
