"""Seeded random shapes and rates for the ZDT (fused where eligible, staged otherwise)
against the FP64 oracle on a few sampled columns, rate-block subsets against the full run,
and a large rate count.  Tolerance: relative L-infinity 1e-5 against FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(rng):
    Nf = int(2 ** rng.integers(12, 21)) if rng.random() < 0.8 else int(rng.integers(500, 5000))
    Nt = int(rng.integers(1, 65))
    Nr = int(rng.integers(1, 200))
    dr = float(np.float32(rng.choice([1 / 16, 1 / 8, 0.25, 1 / 15, 0.1])))
    r0 = float(np.float32(rng.uniform(-6, 2)))
    return Nf, Nt, Nr, r0, dr


@pytest.mark.parametrize("seed", range(12))
def test_random_shape_vs_fp64(fdr, oracle, seed):
    rng = np.random.default_rng(1000 + seed)
    Nf, Nt, Nr, r0, dr = _case(rng)
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 10.0, 30.0, 2.0, seed=seed)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr)
    out = fdr.zdtfdr(ws).cpu().numpy()
    cols = sorted(set([0, Nr - 1, int(rng.integers(0, Nr))]))
    rates = [float(np.float32(r0)) + j * float(np.float32(dr)) for j in cols]
    err = oracle.rel_linf(out[:, cols], oracle.fdr_truth(spec, rates))
    assert err < 1e-5, (Nf, Nt, Nr, r0, dr, ws.fused, err)
    if ws.fused and Nr >= 16:
        nb = Nr // 8
        blocks = rng.choice(nb, size=min(3, nb), replace=False).tolist()
        sub = fdr.fortran_empty(Nf, 8 * len(blocks))
        fdr.zdtfdr_blocks_(sub, ws, spec, blocks)
        cols2 = [8 * b + u for b in blocks for u in range(8)]
        assert np.array_equal(sub.cpu().numpy(), out[:, cols2])


def test_many_rates(fdr, oracle):
    """1025 rates at Nf = 2^20 (513 rate pairs of W, about 4.3 GB)."""
    Nf, Nt, Nr = 1 << 20, 16, 1025
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 4, 10.0, 30.0, 4.0, seed=77)
    ws = fdr.ZDTWorkspace(spec, -32.0, 1 / 16, Nr)
    assert ws.fused
    out = fdr.zdtfdr(ws)
    cols = [0, 511, 1024]
    got = out[:, cols].cpu().numpy()
    err = oracle.rel_linf(got, oracle.fdr_truth(spec, [-32.0 + j / 16 for j in cols]))
    assert err < 1e-5, err


@pytest.mark.parametrize("seed", range(8))
def test_random_shared_memory_f_and_snr_search(fdr, oracle, seed):
    """16 < Nt <= 64 (F in shared memory; the warp-specialised czt kernel at 256 or 512 bins
    per CTA): FP64 on sampled columns, rate blocks bit for bit against the full run, and the
    fused snr proto-hit search (pairwise fdrstats, leaf-gated) equal to the oracle's hits."""
    rng = np.random.default_rng(70000 + seed)
    Nf = int(2 ** rng.integers(12, 19))
    Nt = int(rng.integers(17, 65))
    Nr = int(rng.integers(1, 120))
    dr = float(np.float32(rng.choice([1 / 16, 1 / 8, 0.25, 0.1])))
    r0 = float(np.float32(rng.uniform(-6, 2)))
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 10.0, 30.0, 2.0, seed=seed)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr)
    assert ws.fused
    out = fdr.zdtfdr(ws).cpu().numpy()
    cols = sorted(set([0, Nr - 1, int(rng.integers(0, Nr))]))
    rates = [float(np.float32(r0)) + j * float(np.float32(dr)) for j in cols]
    err = oracle.rel_linf(out[:, cols], oracle.fdr_truth(spec, rates))
    assert err < 1e-5, (Nf, Nt, Nr, r0, dr, err)
    if Nr >= 16:
        nb = Nr // 8
        blocks = rng.choice(nb, size=min(3, nb), replace=False).tolist()
        sub = fdr.fortran_empty(Nf, 8 * len(blocks))
        fdr.zdtfdr_blocks_(sub, ws, spec, blocks)
        assert np.array_equal(sub.cpu().numpy(), out[:, [8 * b + u for b in blocks for u in range(8)]])
    snr = [2, 3.5, np.float32(2.5)][seed % 3]  # Int, Float64 and Float32 snr
    dest = fdr.fortran_empty(Nf, Nr)
    hits = fdr.zdtfdr_protohits_(dest, ws, spec, threshold=snr, snr=True)
    assert np.array_equal(hits, oracle.findprotohits(dest.cpu().numpy(), snr, snr=True))
