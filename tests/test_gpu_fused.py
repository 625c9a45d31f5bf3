"""GPU parity tests of the fused ZDT kernels (power-of-two Nf, Nt <= 64) against the staged
kernels and the CPU oracle.

Tolerances (relative L-infinity): 1e-4 vs FP64 (the accuracy bound of the FDR; the fused path reduces
chirp phases exactly and is typically ~1e-6); 2e-5 vs the staged kernels and the FP32
mirror, which carry the reference's Float32 phase-argument rounding (~5e-6 at Nf=2^20).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spec(oracle, Nf, Nt, seed, ntones=3):
    spec, _ = oracle.synth_spectrogram(Nf, Nt, ntones, 20.0, 20.0, 4.0, seed=seed)
    return spec


@pytest.mark.parametrize("Nf,Nt,r0,dr,Nr", [
    (4096, 16, -4.0, 0.25, 33), (4096, 7, 1.5, -0.125, 8), (8192, 16, -2.0, 1 / 16, 5),
    (2 ** 13, 2, 0.0, 0.5, 1), (2 ** 15, 15, -3.0, 0.1, 2), (2 ** 17, 16, -4.0, 0.25, 33),
    (2 ** 21, 4, -1.0, 0.25, 9), (2 ** 22, 2, 0.5, 1.0, 3),
    # F in shared memory (16 < Nt <= 64)
    (4096, 32, -2.0, 1 / 16, 65), (2 ** 14, 17, -1.0, 0.25, 9), (2 ** 16, 64, -2.0, 1 / 16, 65),
    (2 ** 18, 33, -8.0, 1 / 16, 257), (2 ** 20, 64, -2.0, 1 / 16, 3),
    # 32 < Nt <= 64 at 2^20 and 2^21: two-CTA cluster czt kernel
    (2 ** 20, 40, 1.0, 0.25, 17), (2 ** 21, 36, -2.0, 1 / 16, 3)])
def test_fused_vs_truth_and_staged(fdr, oracle, Nf, Nt, r0, dr, Nr):
    spec = _spec(oracle, Nf, Nt, seed=Nf + Nt)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr)
    assert ws.fused
    out = fdr.zdtfdr(ws).cpu().numpy()
    rates = [float(np.float32(r0)) + j * float(np.float32(dr)) for j in range(Nr)]
    cols = list(range(Nr)) if Nf <= 2 ** 17 else [0, Nr - 1]
    truth = oracle.fdr_truth(spec, [rates[j] for j in cols])
    err = oracle.rel_linf(out[:, cols], truth)
    assert err < 1e-5, err
    st = fdr.ZDTWorkspace(spec, r0, dr, Nr, staged_only=True)
    assert not st.fused
    assert oracle.rel_linf(out, fdr.zdtfdr(st).cpu().numpy()) < 2e-5


def test_config2_fused(fdr, oracle):
    """Nf=2^20, Nt=16, rates -4:1/16:4 (129) -- the benchmark workload.  All 129 columns
    against the oracle's FP32 restatement of the reference's stage sequence (2e-5 relative
    L-infinity: the reference's Float32 phase arguments err by ~5e-6 here), 17 columns
    against the FP64 exact-phase truth (1e-5), the integer rates against intfdr."""
    import os
    spec, _ = oracle.synth_spectrogram(2 ** 20, 16, 20, 8.0, 50.0, 4.0, seed=2000)
    ws = fdr.ZDTWorkspace(spec, -4.0, 1 / 16, 129)
    assert ws.fused and ws.Nl == 144
    out = fdr.zdtfdr(ws).cpu().numpy()
    mirror = oracle.zdtfdr(spec, -4.0, 1 / 16, 129, workers=os.cpu_count())
    err32 = oracle.rel_linf(out, mirror)
    assert err32 < 2e-5, err32
    cols = list(range(0, 129, 8)) + [37, 100]
    truth = oracle.fdr_truth(spec, [-4.0 + j / 16 for j in cols])
    err = oracle.rel_linf(out[:, cols], truth)
    assert err < 1e-5, err
    # integer drift rates are exact circular-shift sums
    icols = [0, 16, 32, 48, 64, 80, 96, 112, 128]
    ref = oracle.intfdr(spec, [-4 + j // 16 for j in icols])
    assert oracle.rel_linf(out[:, icols], ref) < 1e-5
    # and the library's staged kernels (the reference's FP32 stage sequence) agree too
    staged = fdr.zdtfdr(fdr.ZDTWorkspace(spec, -4.0, 1 / 16, 129, staged_only=True)).cpu().numpy()
    assert oracle.rel_linf(out, staged) < 2e-5


def test_fused_windows_and_batches(fdr, oracle):
    spec = _spec(oracle, 2 ** 14, 16, seed=5)
    ws = fdr.ZDTWorkspace(spec, -2.0, 0.25, 17)
    st = fdr.ZDTWorkspace(spec, -2.0, 0.25, 17, staged_only=True)
    for w in ("hamming", lambda n, N: 1.0 - n / N):
        a = fdr.zdtfdr(ws, w=w).cpu().numpy()
        b = fdr.zdtfdr(st, w=w).cpu().numpy()
        assert oracle.rel_linf(a, b) < 2e-5
    dests = [fdr.fortran_empty(2 ** 14, 17) for _ in range(3)]
    fdr.zdtfdr_(dests, ws, r0=[-6.0, -1.75, 2.5])
    for d, r0 in zip(dests, [-6.0, -1.75, 2.5]):
        truth = oracle.fdr_truth(spec, [r0 + 0.25 * j for j in range(17)])
        assert oracle.rel_linf(d.cpu().numpy(), truth) < 1e-5


@pytest.mark.parametrize("Nf,Nt,Nr", [(2 ** 16, 32, 41), (2 ** 17, 64, 65), (2 ** 15, 24, 9), (2 ** 19, 20, 17),
                                       (2 ** 20, 48, 9)])
def test_fused_windows_and_batches_shared_memory_f(fdr, oracle, Nf, Nt, Nr):
    """16 < Nt <= 64 with 256 or 512 bins per czt CTA (the warp-specialised czt kernel, and
    the two-CTA cluster kernel at Nf = 2^20 with Nt > 32): Hamming and custom windows and an
    r0 list against the staged kernels and FP64."""
    P, Q = fdr.fused_split(Nf, Nt, Nr)
    assert Q in (256, 512)
    spec = _spec(oracle, Nf, Nt, seed=3 * Nf + Nt)
    ws = fdr.ZDTWorkspace(spec, -2.0, 1 / 16, Nr)
    st = fdr.ZDTWorkspace(spec, -2.0, 1 / 16, Nr, staged_only=True)
    for w in ("hamming", lambda n, N: 1.0 - n / N):
        a = fdr.zdtfdr(ws, w=w).cpu().numpy()
        b = fdr.zdtfdr(st, w=w).cpu().numpy()
        assert oracle.rel_linf(a, b) < 2e-5
    dests = [fdr.fortran_empty(Nf, Nr) for _ in range(2)]
    fdr.zdtfdr_(dests, ws, r0=[-3.0, 0.5])
    for d, r0 in zip(dests, [-3.0, 0.5]):
        cols = [0, Nr // 2, Nr - 1]
        truth = oracle.fdr_truth(spec, [r0 + j / 16 for j in cols])
        assert oracle.rel_linf(d.cpu().numpy()[:, cols], truth) < 1e-5


def test_fused_input_then_staged_stages(fdr, oracle):
    """input! through the fused path, then the staged stages read F (rebuilt from the fused
    input stage) -- equal to a staged-only workspace's F."""
    spec = _spec(oracle, 2 ** 15, 16, seed=9)
    ws = fdr.ZDTWorkspace(spec, -1.0, 0.5, 5)
    st = fdr.ZDTWorkspace(spec, -1.0, 0.5, 5, staged_only=True)
    F1, F2 = ws.F.cpu().numpy(), st.F.cpu().numpy()
    assert np.abs(F1 - F2).max() / np.abs(F2).max() < 1e-6
    fdr.zdtfdr_nodest_(ws)
    d = fdr.fortran_empty(2 ** 15, 5)
    fdr.output_(d, ws)
    truth = oracle.fdr_truth(spec, [-1.0 + 0.5 * j for j in range(5)])
    assert oracle.rel_linf(d.cpu().numpy(), truth) < 1e-5


def test_fused_phase_fallback(fdr, oracle):
    """A rate step whose exact phase needs more than 62 bits runs the staged kernels."""
    spec = _spec(oracle, 4096, 8, seed=13)
    dr = 2.0 ** -60
    ws = fdr.ZDTWorkspace(spec, 1.0, dr, 3)
    out = fdr.zdtfdr(ws).cpu().numpy()
    truth = oracle.fdr_truth(spec, [1.0, 1.0 + dr, 1.0 + 2 * dr])
    assert oracle.rel_linf(out, truth) < 1e-5


@pytest.mark.parametrize("Nf,staged", [(2 ** 16, False), (2 ** 16, True), (2 ** 20, False), (3000, False)])
def test_fused_protohit_scan(fdr, oracle, Nf, staged):
    """zdtfdr! + findprotohits with the fused scan: hits and threshold equal the oracle's
    Float32 fdrstats / fdrdenormalize on the same FDR."""
    spec, _ = oracle.synth_spectrogram(Nf, 16, 8, 8.0, 50.0, 4.0, seed=Nf + 3)
    Nr = 33
    ws = fdr.ZDTWorkspace(spec, -4.0, 0.25, Nr, staged_only=staged)
    dests = [fdr.fortran_empty(Nf, Nr) for _ in range(2)]
    hits, thr = fdr.zdtfdr_protohits_(dests, ws, r0=[-4.0, 4.25], threshold=10.0, snr=True,
                                      return_threshold=True)
    mats = [d.cpu().numpy() for d in dests]
    m, s = oracle.fdrstats(mats)
    assert thr == oracle.fdrdenormalize(10.0, m, s)
    assert np.array_equal(hits, oracle.findprotohits(mats, 10.0, snr=True))
    sep, thr2 = fdr.findprotohits(dests, 10.0, snr=True, return_threshold=True)
    assert thr2 == thr and np.array_equal(sep, hits)
    # absolute threshold (no statistics)
    hits_abs = fdr.zdtfdr_protohits_(dests, ws, r0=[-4.0, 4.25], threshold=40.0, snr=False)
    assert np.array_equal(hits_abs, oracle.findprotohits(mats, 40.0))


@pytest.mark.parametrize("Nf,Nt,r0,dr,Nr,blocks", [
    (2 ** 16, 16, -8.0, 1 / 16, 256, [5, 0, 31, 3, 3]),
    (2 ** 12, 7, -2.0, 0.25, 24, [2, 0]),
    (2 ** 15, 32, -4.0, 1 / 16, 128, [15, 1, 8]),
    (2 ** 20, 16, -8.0, 1 / 16, 256, [0, 17, 18, 31])])
def test_rate_blocks_match_full_run(fdr, oracle, Nf, Nt, r0, dr, Nr, blocks):
    """zdtfdr over a subset of 8-rate blocks in one pass equals the same columns of the
    full run bit for bit, and its proto-hit scan equals findprotohits of its columns."""
    spec = _spec(oracle, Nf, Nt, seed=Nf + 7 * Nt, ntones=5)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr)
    assert ws.fused
    full = fdr.zdtfdr(ws).cpu().numpy()
    dest = fdr.fortran_empty(Nf, 8 * len(blocks))
    fdr.zdtfdr_blocks_(dest, ws, spec, blocks)
    cols = [8 * b + u for b in blocks for u in range(8)]
    got = dest.cpu().numpy()
    assert np.array_equal(got, full[:, cols])
    hits, thr = fdr.zdtfdr_blocks_protohits_(dest, ws, spec, blocks, threshold=8.0, snr=True,
                                             return_threshold=True)
    m, s = oracle.fdrstats(got)
    assert thr == oracle.fdrdenormalize(8.0, m, s)
    assert np.array_equal(hits, oracle.findprotohits(got, thr))


def test_rate_blocks_argument_errors(fdr, oracle):
    spec = _spec(oracle, 4096, 16, seed=1)
    ws = fdr.ZDTWorkspace(spec, -2.0, 0.25, 16)
    with pytest.raises(fdr.FDRError):
        fdr.zdtfdr_blocks_(fdr.fortran_empty(4096, 8), ws, spec, [2])  # rates 16..23 > Nr
    with pytest.raises(fdr.FDRError):
        fdr.zdtfdr_blocks_(fdr.fortran_empty(4096, 24), ws, spec, [0, 1, 0])  # > Nr/8 blocks
    st = fdr.ZDTWorkspace(spec, -2.0, 0.25, 16, staged_only=True)
    with pytest.raises(fdr.FDRError):
        fdr.zdtfdr_blocks_(fdr.fortran_empty(4096, 8), st, spec, [0])


def test_tma_output_matches_register_output(fdr, oracle, monkeypatch):
    """The TMA-fed output pass for P = 1024 writes the same FDR, bit for bit, as the
    register-load output kernel (FDR_NO_TMA=1) with the same 32 x 32 split, with and without
    the fused proto-hit statistics (odd Nt too), and reports no fault."""
    for Nf, Nt, Nr in ((1 << 19, 16, 129), (1 << 18, 40, 33), (1 << 19, 15, 9)):
        spec = _spec(oracle, Nf, Nt, seed=Nf + Nt + 5)
        ws = fdr.ZDTWorkspace(spec, -4.0, 1 / 16, Nr)
        a = fdr.zdtfdr(ws).cpu().numpy()
        ha, ta = fdr.zdtfdr_protohits_(fdr.fortran_empty(Nf, Nr), ws, spec, threshold=8.0,
                                       return_threshold=True)
        fdr.fdrsynchronize()
        monkeypatch.setenv("FDR_NO_TMA", "1")
        b = fdr.zdtfdr(ws).cpu().numpy()
        hb, tb = fdr.zdtfdr_protohits_(fdr.fortran_empty(Nf, Nr), ws, spec, threshold=8.0,
                                       return_threshold=True)
        monkeypatch.delenv("FDR_NO_TMA")
        assert np.array_equal(a, b)
        assert ta == tb and np.array_equal(ha, hb)


@pytest.mark.parametrize("Nf,Nt,Nr", [(1 << 20, 16, 129), (1 << 21, 16, 17), (1 << 20, 15, 9),
                                      (1 << 20, 24, 33)])
def test_tma_output_p2048(fdr, oracle, monkeypatch, Nf, Nt, Nr):
    """The TMA-fed output pass for P = 2048 (64 x 32 split, the 64-point DFT shared by lane
    pairs): FDR within float32 rounding of the shared-memory FFT output kernel
    (FDR_NO_TMA=1) and of the FP64 direct sums on sampled columns, the proto-hits of that FDR
    at the kernel's threshold and no fault."""
    spec = _spec(oracle, Nf, Nt, seed=Nf + Nt + 7)
    ws = fdr.ZDTWorkspace(spec, -4.0, 1 / 16, Nr)
    a = fdr.zdtfdr(ws).cpu().numpy()
    ha, ta = fdr.zdtfdr_protohits_(fdr.fortran_empty(Nf, Nr), ws, spec, threshold=8.0,
                                   return_threshold=True)
    fdr.fdrsynchronize()
    monkeypatch.setenv("FDR_NO_TMA", "1")
    b = fdr.zdtfdr(ws).cpu().numpy()
    monkeypatch.delenv("FDR_NO_TMA")
    scale = np.abs(b).max()
    assert np.abs(a - b).max() <= 2e-6 * scale
    cols = sorted({0, Nr // 2, Nr - 1})
    truth = oracle.fdr_truth(spec, [-4.0 + j / 16 for j in cols])
    assert oracle.rel_linf(a[:, cols], truth) < 1e-5
    m, sd = oracle.fdrstats(a)
    assert ta == oracle.fdrdenormalize(8.0, m, sd)
    assert np.array_equal(ha, oracle.findprotohits(a, ta))


def test_bounded_wait_fault_is_reported(fdr, oracle):
    """A bounded mbarrier wait that runs out (the self-test kernel waits on a barrier that
    nothing completes, 10 ms) raises the fault flag; fdr_synchronize reports it once as
    FDR_ERR_CUDA, and the device stays usable: the next ZDT is correct."""
    import ctypes as C
    fdr._lib.check(fdr._lib.lib().fdr_selftest_bounded_wait(10_000_000, C.c_void_p(None)))
    with pytest.raises(fdr.FDRError, match="timed out"):
        fdr.fdrsynchronize()
    fdr.fdrsynchronize()  # reported once, then cleared
    spec = _spec(oracle, 1 << 20, 16, seed=99)
    ws = fdr.ZDTWorkspace(spec, -4.0, 1 / 16, 9)
    out = fdr.zdtfdr(ws).cpu().numpy()
    truth = oracle.fdr_truth(spec, [-4.0, -3.5])
    assert oracle.rel_linf(out[:, [0, 8]], truth) < 1e-5
    fdr.fdrsynchronize()


@pytest.mark.parametrize("Nf,Nt,Nr,staged", [(1 << 12, 16, 33, False), (1 << 12, 65, 33, False),
                                            (1 << 12, 16, 33, True), (3000, 16, 9, False),
                                            (1 << 20, 16, 129, False)])
def test_workspace_path_matches_fused_split(fdr, oracle, Nf, Nt, Nr, staged):
    """A workspace runs the fused kernels exactly when the host planner returns a split."""
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 1, 20.0, 20.0, 2.0, seed=Nf + Nt)
    ws = fdr.ZDTWorkspace(spec, -2.0, 1 / 16, Nr, staged_only=staged)
    assert ws.fused == (fdr.fused_split(Nf, Nt, Nr, staged_only=staged) is not None)
