"""findprotohits(fdr, snr; snr=true) against the oracle's Float32 restatement of fdrstats
and fdrdenormalize (src/fdrutils.jl:39-50, 104-107, 148-154), at the two benchmark shapes:
the library's own FDR, with FDR values planted one ulp either side of the reference
threshold (for an Int snr the threshold and the comparison are Float32, for a Float64 snr
they are Float64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONFIGS = {
    # (Nf, Nt, ntones, snr_lo, snr_hi, rmax, r0, dr, Nr)
    1: (65536, 16, 3, 20.0, 20.0, 4.0, -4.0, 0.25, 33),
    2: (1 << 20, 16, 20, 8.0, 50.0, 4.0, -4.0, 1 / 16, 129),
}


def _bracket(oracle, thr):
    """(below, at_or_above): the Float32 values just below and at/above the threshold."""
    if isinstance(thr, np.float32):
        return np.nextafter(thr, np.float32(-np.inf)), thr
    f = np.float32(thr)
    if float(f) < thr:
        return f, np.nextafter(f, np.float32(np.inf))
    if float(f) > thr:
        return np.nextafter(f, np.float32(-np.inf)), f
    return np.nextafter(f, np.float32(-np.inf)), f


@pytest.mark.parametrize("cfg", [1, 2])
def test_snr_threshold_parity_with_planted_ulps(fdr, oracle, cfg):
    Nf, Nt, nt, lo, hi, rmax, r0, dr, Nr = CONFIGS[cfg]
    spec, _ = oracle.synth_spectrogram(Nf, Nt, nt, lo, hi, rmax, seed=1000 * cfg)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr)
    dest = fdr.fortran_empty(Nf, Nr)
    for snr in (10, 10.0):
        # the fused scan on the library's FDR gives the oracle's hits for that FDR
        hits_fused, thr_fused = fdr.zdtfdr_protohits_(dest, ws, spec, threshold=snr, snr=True,
                                                      return_threshold=True)
        F = dest.cpu().numpy()
        m, s = oracle.fdrstats(F)
        thr = oracle.fdrdenormalize(snr, m, s)
        assert thr_fused == float(thr)
        assert np.array_equal(hits_fused, oracle.findprotohits(F, snr, snr=True))

        # plant values one ulp either side of the threshold in a column that is neither the
        # first (m) nor the one of least standard deviation (s), so m and s stay the same
        stds = oracle._std32_columns(F)
        jp = next(j for j in np.argsort(stds)[::-1] if j not in (0, int(np.argmin(stds))))
        below, above = _bracket(oracle, thr)
        rows = [Nf // 7, Nf // 3, (2 * Nf) // 3]
        P = F.copy()
        P[rows[0], jp] = below
        P[rows[1], jp] = above
        P[rows[2], jp] = np.nextafter(above, np.float32(np.inf))
        assert oracle.fdrstats(P) == (m, s)
        g = fdr.as_device_f32(P)
        hits, thr_g = fdr.findprotohits(g, snr, snr=True, return_threshold=True)
        assert thr_g == float(thr)
        ref = oracle.findprotohits(P, snr, snr=True)
        assert np.array_equal(hits, ref)
        planted = {(r, int(jp)) for r in rows}
        got = {(int(i), int(j)) for i, j in hits} & planted
        assert got == {(rows[1], int(jp)), (rows[2], int(jp))}
        del g


def test_fast_stats_option(fdr, oracle):
    """FDR_ZDT_FAST_STATS: float64 moments accumulated by the output kernels; m and s agree
    with the float64 restatement, and the hits with findprotohits at that threshold."""
    Nf, Nt, nt, lo, hi, rmax, r0, dr, Nr = CONFIGS[1]
    spec, _ = oracle.synth_spectrogram(Nf, Nt, nt, lo, hi, rmax, seed=1001)
    ws = fdr.ZDTWorkspace(spec, r0, dr, Nr, fast_stats=True)
    dest = fdr.fortran_empty(Nf, Nr)
    hits, thr = fdr.zdtfdr_protohits_(dest, ws, spec, threshold=10.0, snr=True, return_threshold=True)
    F = dest.cpu().numpy()
    m64, s64 = oracle.fdrstats_f64(F)
    ref_thr = 10.0 * float(np.float32(s64)) + float(np.float32(m64))
    assert abs(thr - ref_thr) <= 1e-6 * ref_thr
    assert np.array_equal(hits, oracle.findprotohits(F, thr))
