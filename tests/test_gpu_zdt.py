"""GPU parity tests of the ZDT path (zdtfdr.jl) through the C ABI against the CPU oracle.

Tolerances (relative L-infinity, max|a-b| / max|b|):
  * vs the FP64 oracle: 1e-4 (the accuracy bound of the FDR); the library is typically ~1e-6 at
    Nf <= 65536 and ~5e-6 at Nf = 2^20 with the reference's Float32 phase arguments.
  * vs the FP32 mirror of the reference: 2e-5 (both carry float32 rounding of their own
    FFTs; the phase arguments are the same Float32 values).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-4
TOL_MIRROR = 2e-5


def _spec(oracle, Nf, Nt, seed, ntones=3, rmax=4.0):
    spec, _ = oracle.synth_spectrogram(Nf, Nt, ntones, 20.0, 20.0, rmax, seed=seed)
    return spec


def test_known_answers(fdr, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    exp = np.array(golden["fdr_expected"], dtype=np.float32)
    for kw in ({}, {"exact_phase": True}, {"staged_only": True}):
        ws = fdr.ZDTWorkspace(d, range(-1, 2), **kw)
        assert ws.Nl == 4
        np.testing.assert_allclose(fdr.zdtfdr(ws).cpu().numpy(), exp, atol=2e-6)


@pytest.mark.parametrize("Nf,Nt,r0,dr,Nr", [(4096, 16, -4.0, 0.25, 33), (1000, 7, 2.0, -0.5, 9),
                                           (375, 5, -1.0, 0.125, 17), (65536, 16, -4.0, 0.25, 33)])
def test_staged_buffers_match_mirror(fdr, oracle, Nf, Nt, r0, dr, Nr):
    spec = _spec(oracle, Nf, Nt, seed=Nf + Nt)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr, staged_only=True)
    mw = oracle.ZDTWorkspace(spec, r0, dr, Nr)
    assert ws.Nl == mw.Nl and ws.K == mw.K
    scale = np.abs(mw.F).max()
    assert np.abs(ws.F.cpu().numpy() - mw.F).max() / scale < 1e-6
    vs = np.abs(mw.V).max()
    assert np.abs(ws.V.cpu().numpy() - mw.V).max() / vs < 2e-6
    fdr.preprocess_(ws)
    mw.preprocess()
    assert np.abs(ws.Y.cpu().numpy() - mw.Y).max() / scale < 1e-6
    fdr.convolve_(ws)
    mw.convolve()
    ys = np.abs(mw.Y).max()
    assert np.abs(ws.Y.cpu().numpy() - mw.Y).max() / ys < 5e-6
    fdr.postprocess_(ws)
    mw.postprocess()
    assert np.abs(ws.Ys.cpu().numpy() - mw.Y[:, :Nr]).max() / ys < 5e-6
    dest = fdr.fortran_empty(Nf, Nr)
    fdr.output_(dest, ws)
    out = dest.cpu().numpy()
    assert oracle.rel_linf(out, mw.output()) < TOL_MIRROR


@pytest.mark.parametrize("exact", [False, True])
def test_config1_vs_fp64(fdr, oracle, exact):
    """Nf=65536, Nt=16, rates -4:0.25:4 (33), 3 tones at SNR 20."""
    spec, _ = oracle.synth_spectrogram(65536, 16, 3, 20.0, 20.0, 4.0, seed=1000)
    ws = fdr.ZDTWorkspace(spec, -4.0, 0.25, 33, exact_phase=exact)
    out = fdr.zdtfdr(ws).cpu().numpy()
    truth = oracle.fdr_truth(spec, [-4.0 + 0.25 * j for j in range(33)])
    err = oracle.rel_linf(out, truth)
    assert err < 1e-5, err
    mirror = oracle.zdtfdr(spec, -4.0, 0.25, 33)
    assert oracle.rel_linf(out, mirror) < TOL_MIRROR


def test_integer_rates_equal_intfdr(fdr, oracle):
    spec = _spec(oracle, 8192, 16, seed=21)
    ws = fdr.ZDTWorkspace(spec, -4.0, 1.0, 9)
    out = fdr.zdtfdr(ws).cpu().numpy()
    ref = oracle.intfdr(spec, list(range(-4, 5)))
    assert oracle.rel_linf(out, ref) < 1e-5


def test_r0_iterator_and_batches(fdr, oracle):
    """zdtfdr!(dests, ws; r0=iterator) reuses V across batches (zdtfdr.jl:354)."""
    spec = _spec(oracle, 4096, 16, seed=22)
    ws = fdr.ZDTWorkspace(spec, -4.0, 0.25, 17)
    dests = [fdr.fortran_empty(4096, 17) for _ in range(3)]
    r0s = [-4.0, 0.25, 4.5]
    fdr.zdtfdr_(dests, ws, r0=r0s)
    for d, r0 in zip(dests, r0s):
        truth = oracle.fdr_truth(spec, [r0 + 0.25 * j for j in range(17)])
        assert oracle.rel_linf(d.cpu().numpy(), truth) < 1e-5
    # scalar r0 cycles over all dests
    fdr.zdtfdr_(dests[:2], ws, r0=1.0)
    np.testing.assert_array_equal(dests[0].cpu().numpy(), dests[1].cpu().numpy())


def test_new_spectrogram_via_execute(fdr, oracle):
    s1 = _spec(oracle, 4096, 16, seed=31)
    s2 = _spec(oracle, 4096, 16, seed=32)
    ws = fdr.ZDTWorkspace(s1, -2.0, 0.25, 17)
    out = fdr.zdtfdr(ws, s2).cpu().numpy()
    truth = oracle.fdr_truth(s2, [-2.0 + 0.25 * j for j in range(17)])
    assert oracle.rel_linf(out, truth) < 1e-5
    # the staged stages see the new spectrogram too (F follows input!)
    fdr.zdtfdr_nodest_(ws)
    dest = fdr.fortran_empty(4096, 17)
    fdr.output_(dest, ws)
    assert oracle.rel_linf(dest.cpu().numpy(), truth) < 1e-5


@pytest.mark.parametrize("w", ["hamming", "custom"])
def test_windows(fdr, oracle, w):
    spec = _spec(oracle, 4096, 16, seed=41)
    ws = fdr.ZDTWorkspace(spec, -2.0, 0.25, 17)
    mw = oracle.ZDTWorkspace(spec, -2.0, 0.25, 17)
    fn = (lambda n, N: 0.5 + 0.5 * np.cos(2 * np.pi * n / N)) if w == "custom" else "hamming"
    out = fdr.zdtfdr(ws, w=fn).cpu().numpy()
    ref = mw.zdtfdr(window=fn)
    assert oracle.rel_linf(out, ref) < TOL_MIRROR
    with pytest.raises(fdr.FDRError):
        fdr.zdtfdr(ws, w="blackman")


@pytest.mark.parametrize("Nf,Nt,Nr", [(3, 2, 3), (1000, 7, 1), (1024, 1, 5), (7 * 512, 3, 10),
                                      (2 ** 14 * 3, 16, 33)])
def test_edge_shapes(fdr, oracle, Nf, Nt, Nr):
    spec = _spec(oracle, Nf, Nt, seed=Nf * 7 + Nt, ntones=1, rmax=2.0)
    r0, dr = -1.5, 0.25
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr)
    out = fdr.zdtfdr(ws).cpu().numpy()
    truth = oracle.fdr_truth(spec, [r0 + dr * j for j in range(Nr)])
    assert oracle.rel_linf(out, truth) < 1e-5


def test_descending_rates_heavytest_standin(fdr, oracle):
    """test/heavytests.jl stand-in: rates 0:-0.25:-5 (dr < 0), peak at (54, 10)."""
    rng = np.random.Generator(np.random.PCG64(11))
    Nf, Nt = 150, 16
    spec = rng.exponential(1.0, size=(Nf, Nt)).astype(np.float32)
    for t in range(Nt):
        c = 54 - 2.5 * t
        lo = int(np.floor(c))
        f = c - lo
        spec[lo % Nf, t] += 40 * (1 - f)
        spec[(lo + 1) % Nf, t] += 40 * f
    ws = fdr.ZDTWorkspace(spec, 0.0, -0.25, 21)
    out = fdr.zdtfdr(ws).cpu().numpy()
    assert np.unravel_index(np.argmax(out), out.shape) == (54, 10)


def test_errors(fdr, oracle):
    spec = _spec(oracle, 1024, 4, seed=3)
    ws = fdr.ZDTWorkspace(spec, 0.0, 1.0, 3)
    with pytest.raises(fdr.FDRError):
        fdr.output_(fdr.fortran_empty(1024, 4), ws)   # wrong dest size
    with pytest.raises(fdr.FDRError):
        fdr.input_(ws, _spec(oracle, 1024, 5, seed=4))  # wrong spectrogram size
    with pytest.raises(fdr.FDRError) as e:
        fdr.ZDTWorkspace(_spec(oracle, 67 * 4, 4, seed=5), 0.0, 1.0, 3)
    assert e.value.status == fdr._lib.FDR_ERR_UNSUPPORTED_SIZE


def test_info_and_show(fdr, oracle):
    spec = _spec(oracle, 2048, 16, seed=6)
    ws = fdr.ZDTWorkspace(spec, -4.0, 0.25, 33)
    assert (ws.Nf, ws.Nt, ws.Nr, ws.Nl, ws.K) == (2048, 16, 33, 48, 1025)
    assert ws.r0 == -4.0 and ws.dr == 0.25
    assert "Nl=48" in repr(ws)
    assert ws.nbytes() >= 8 * 1025 * (16 + 2 * 48)
    np.testing.assert_array_equal(fdr.driftrates(ws), np.float32(-4 + 0.25 * np.arange(33)))
