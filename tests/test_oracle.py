"""CPU tests of the oracle itself: pinned to the reference's known answers
(test/runtests.jl:5-32) and cross-checked between its FP32 mirror and FP64 tiers."""
from fractions import Fraction

import numpy as np
import pytest


def test_known_answers_intshift_intfdr(oracle, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    assert np.array_equal(oracle.intshift(d, golden["intshift_rate"]),
                          np.array(golden["intshift_expected"], dtype=np.float32))
    # runtests.jl:20 compares with `==`
    assert np.array_equal(oracle.intfdr(d, golden["rates"]),
                          np.array(golden["fdr_expected"], dtype=np.float32))


def test_known_answers_fftfdr(oracle, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    ws = oracle.fftfdr_workspace(d)
    np.testing.assert_allclose(oracle.fdshift(ws, 1), np.array(golden["intshift_expected"]),
                               atol=1e-6)
    np.testing.assert_allclose(oracle.fftfdr(ws, golden["rates"]),
                               np.array(golden["fdr_expected"]), atol=1e-6)


def test_known_answers_zdtfdr(oracle, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    ws = oracle.ZDTWorkspace(d, -1, 1, 3)
    assert ws.Nl == 4  # nextprod((2,3,5), 2+3-1)
    np.testing.assert_allclose(ws.zdtfdr(), np.array(golden["fdr_expected"]), atol=1e-6)


def test_truth_known_answers(oracle, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    np.testing.assert_allclose(oracle.fdr_truth(d, [-1.0, 0.0, 1.0]),
                               np.array(golden["fdr_expected"]), atol=1e-12)


def test_truth_equals_circular_shift_at_integer_rates(oracle):
    spec, _ = oracle.synth_spectrogram(1024, 8, 2, 20, 20, 3, seed=1)
    rates = [-3.0, -1.0, 0.0, 2.0, 3.0]
    shifts = [[int(r * t) for t in range(8)] for r in rates]
    np.testing.assert_allclose(oracle.fdr_truth(spec, rates), oracle.intfdr_f64(spec, shifts),
                               rtol=0, atol=1e-9)


@pytest.mark.parametrize("Nf,Nt,r0,dr,Nr", [(4096, 16, -4.0, 0.25, 33), (1000, 7, 2.0, -0.5, 9),
                                           (375, 5, -1.0, 0.125, 17)])
def test_fp32_zdt_mirror_vs_fp64_truth(oracle, Nf, Nt, r0, dr, Nr):
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 20, 20, 4, seed=Nf)
    out = oracle.zdtfdr(spec, r0, dr, Nr)
    truth = oracle.fdr_truth(spec, [r0 + j * dr for j in range(Nr)])
    assert oracle.rel_linf(out, truth) < 1e-5


def test_fp32_fftfdr_mirror_vs_fp64_truth(oracle):
    spec, _ = oracle.synth_spectrogram(2048, 16, 2, 20, 20, 4, seed=3)
    rates = [-4.0 + 0.25 * j for j in range(33)]
    ws = oracle.fftfdr_workspace(spec)
    assert oracle.rel_linf(oracle.fftfdr(ws, rates), oracle.fdr_truth(spec, rates)) < 1e-5


def test_zdt_equals_intfdr_at_integer_rates(oracle):
    spec, _ = oracle.synth_spectrogram(2048, 16, 3, 20, 20, 3, seed=5)
    out = oracle.zdtfdr(spec, -3.0, 1.0, 7)
    ref = oracle.intfdr(spec, [-3, -2, -1, 0, 1, 2, 3])
    assert oracle.rel_linf(out, ref) < 1e-5


def test_windows_mirror(oracle):
    spec, _ = oracle.synth_spectrogram(512, 8, 1, 20, 20, 2, seed=9)
    ws = oracle.ZDTWorkspace(spec, -2.0, 0.5, 9)
    rect = ws.zdtfdr(window="rect")
    ham = ws.zdtfdr(window="hamming")
    same = ws.zdtfdr(window=lambda n, N: 1.0)
    np.testing.assert_allclose(same, rect, atol=1e-5 * np.abs(rect).max())
    assert not np.allclose(ham, rect)
    with pytest.raises(ValueError):
        ws.zdtfdr(window="blackman")


def test_heavytest_standin_peak(oracle):
    """Stand-in for test/heavytests.jl:9-40 (Voyager-1 data unavailable): a tone starting at
    channel 54 (0-based) drifting -2.5 ch/step, rates 0:-0.25:-5 -> peak at (54, 10)."""
    rng = np.random.Generator(np.random.PCG64(11))
    Nf, Nt = 150, 16
    spec = rng.exponential(1.0, size=(Nf, Nt)).astype(np.float32)
    for t in range(Nt):
        c = 54 - 2.5 * t
        lo = int(np.floor(c))
        f = c - lo
        spec[lo % Nf, t] += 40 * (1 - f)
        spec[(lo + 1) % Nf, t] += 40 * f
    rates = [0.0 - 0.25 * j for j in range(21)]
    for out in (oracle.intfdr(spec, rates),
                oracle.fftfdr(oracle.fftfdr_workspace(spec), rates),
                oracle.zdtfdr(spec, 0.0, -0.25, 21)):
        assert np.unravel_index(np.argmax(out), out.shape) == (54, 10)


def test_zdtutils(oracle):
    assert oracle.calcNl(16, 129) == 144
    assert oracle.calcNl(16, 33) == 48
    assert oracle.calcNl(2, 3) == 4
    assert oracle.growNr(16, 129) == 129
    assert oracle.growNr(16, 30) == 30
    assert oracle.calcNl(16, 129, (2,)) == 256
    assert oracle.estimate_memory(2 ** 20, 16, 129) == 4 * (2 ** 20 * 16 * 4 + 2 ** 20 * 144 * 3
                                                          + 2 ** 20 * 129)


def test_batchrates_properties(oracle):
    for Nt, dh, r1, r2, Nrb in [(16, 1.0, -4.0, None, 360), (16, 0.5, 10.0, -3.0, 50),
                                (32, -0.25, -2.0, 5.0, 40), (17, 0.1, -100.0, 100.0, 360)]:
        batches = oracle.batchrates(Nt, dh, r1, r2, Nrb=Nrb)
        n = len(batches[0])
        assert all(len(b) == n for b in batches)
        assert oracle.growNr(Nt, n) == n
        flat = [r for b in batches for r in b]
        steps = {flat[i + 1] - flat[i] for i in range(len(flat) - 1)}
        assert steps <= {Fraction(1, Nt - 1), Fraction(-1, Nt - 1)}
        lo, hi = (r1, -r1 if r2 is None else r2)
        lo, hi = min(lo, hi), max(lo, hi)
        span = {round(lo / dh), round(hi / dh)}
        covered = {int(r * (Nt - 1)) for r in flat}
        assert span <= covered


def test_proposal_restatement_finite_differences(oracle):
    """The FP64 restatement of the proposal net (the checker of the CUDA gradients) agrees
    with central finite differences of its own loss."""
    rng = np.random.default_rng(0)
    nt, X, B = 3, 20, 2
    n = sum(co * ci * k + co for ci, co, k in oracle.propose_layers(nt))
    p = rng.normal(0, 0.3, n)
    x = rng.normal(0, 1, (B, nt, X))
    lab = (rng.random((B, 16)) < 0.3).astype(float)
    _, g = oracle.propose_loss_and_grad(p, x, lab, nt, half_weights=False)
    eps = 1e-6
    for i in rng.choice(n, 24, replace=False):
        q = p.copy()
        q[i] += eps
        l1, _ = oracle.propose_loss_and_grad(q, x, lab, nt, half_weights=False)
        q[i] -= 2 * eps
        l2, _ = oracle.propose_loss_and_grad(q, x, lab, nt, half_weights=False)
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), 1e-3)


def test_proposal_features_restatement(oracle):
    rng = np.random.default_rng(1)
    Nf, Nt = 1024, 4
    s = -np.log(rng.random((Nf, Nt)))
    p = oracle.propose_features(s, factor=256)
    assert p.shape == (Nt, 4)
    assert np.allclose(p[2, 1], (s[256:512, 2].sum() - 256) / 16)
    lf = oracle.propose_lag_features(s, factor=256, maxlag=8)
    l, b = 3, 2  # lag +3 of bin 2, with wrap-around inside the sum
    ref = sum((s[n, t] - 1) * (s[(n + l) % Nf, t + 1] - 1)
              for n in range(512, 768) for t in range(Nt - 1)) / np.sqrt(256 * (Nt - 1))
    assert np.isclose(lf[l + 8, b], ref)


def test_cluster_restatement_small(oracle):
    """Hand-checked components of the clustering restatement."""
    hits = np.array([[1, 0], [2, 0], [7, 0], [3, 1], [8, 2], [0, 4]])
    labels, cl = oracle.cluster_protohits(hits, 10, 1, 1)
    # (1,0)-(2,0)-(3,1) touch; (7,0) alone ((8,2) is two columns away); (8,2); (0,4)
    assert list(labels) == [0, 0, 1, 0, 2, 3]
    assert [c["count"] for c in cl] == [3, 1, 1, 1]
    assert cl[0]["i_max"] == 3 and cl[0]["j_max"] == 1 and cl[0]["first"] == 0
    labels2, _ = oracle.cluster_protohits(hits, 10, 1, 2)
    assert labels2[2] == labels2[4]  # (7,0)-(8,2) with dj = 2


def test_taylor_restatement_is_a_path_sum(oracle, fdr):
    """The float32 Taylor-tree restatement equals the sum along taylor_shifts' paths (integer
    data: exact), the paths end at channel d and stay near the straight line."""
    rng = np.random.default_rng(2)
    Nf, Nt = 64, 16
    s = rng.integers(0, 50, (Nf, Nt)).astype(np.float32)
    out = oracle.taylor_tree(s, -(Nt - 1), Nt - 1)
    idx = np.arange(Nf)
    worst = 0.0
    for d in range(-(Nt - 1), Nt):
        p = fdr.taylor_shifts(Nt, d)
        assert p[0] == 0 and p[-1] == d
        ref = sum(s[(idx + p[t]) % Nf, t].astype(np.float64) for t in range(Nt))
        assert np.array_equal(out[:, d + Nt - 1], ref.astype(np.float32))
        worst = max(worst, max(abs(p[t] - d * t / (Nt - 1)) for t in range(Nt)))
    assert worst <= 1.0  # within one channel of the straight line (0.67 at Nt = 16)


def _julia_pairwise_literal(x, f=lambda v: v, blk=1024):
    """Element-by-element transliteration of Base.mapreduce_impl (julia base/reduce.jl) in
    numpy float32 scalars, with the sequential leaf loop in its written order."""
    def impl(lo, hi):  # 1-based inclusive
        if lo == hi:
            return f(x[lo - 1])
        if hi - lo < blk:
            v = np.float32(f(x[lo - 1]) + f(x[lo]))
            for i in range(lo + 2, hi + 1):
                v = np.float32(v + f(x[i - 1]))
            return v
        mid = lo + ((hi - lo) >> 1)
        return np.float32(impl(lo, mid) + impl(mid + 1, hi))
    return impl(1, len(x))


@pytest.mark.parametrize("n", [1, 2, 3, 15, 16, 17, 1024, 1025, 2048, 2049, 3000, 8195, 12289])
def test_pairwise_sum32_matches_literal_recursion(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.exponential(1.0, n).astype(np.float32) * np.float32(7.3)
    got = oracle.pairwise_sum32(x)[0]
    assert got.dtype == np.float32
    assert got == _julia_pairwise_literal(x)
    m = np.float32(np.float32(got) / np.float32(n))
    sq = oracle.pairwise_sum32(x, f=lambda v: np.square((v - m).astype(np.float32)))[0]
    lit = _julia_pairwise_literal(x, f=lambda v: np.float32(np.float32(v - m) * np.float32(v - m)))
    assert sq == lit


def test_pairwise_leaves_cover_and_split(oracle):
    for n in [1, 1024, 1025, 5000, 1 << 20, (1 << 20) + 3]:
        lv = oracle.pairwise_leaves(n)
        assert lv[0][0] == 0 and lv[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(lv, lv[1:]))
        assert all(1 <= b - a <= 1024 for a, b in lv)


def test_fdrstats_float32_semantics(oracle):
    rng = np.random.default_rng(5)
    M = rng.exponential(1.0, (3000, 5)).astype(np.float32)
    m, s = oracle.fdrstats(M)
    assert isinstance(m, np.float32) and isinstance(s, np.float32)
    assert m == np.float32(_julia_pairwise_literal(M[:, 0]) / np.float32(3000))
    inv = np.float32(1.0) / np.float32(2999)  # Float32(1 // (n-1))
    stds = []
    for j in range(5):
        mj = np.float32(_julia_pairwise_literal(M[:, j]) / np.float32(3000))
        ss = _julia_pairwise_literal(M[:, j], f=lambda v: np.float32(np.float32(v - mj) ** 2))
        stds.append(np.sqrt(np.float32(ss * inv)))
    assert s == min(stds)
    # float64 statistics agree to float32 rounding
    m64, s64 = oracle.fdrstats_f64(M)
    assert abs(m - m64) <= 4e-7 * m64 and abs(s - s64) <= 4e-7 * s64
    # the iterable form: m from the first matrix, s the minimum over all columns
    m2, s2 = oracle.fdrstats([M[:, :2], M[:, 2:4]])
    assert m2 == m and s2 == min(stds[:4])
    # NaN in any column makes s NaN
    M2 = M.copy()
    M2[7, 3] = np.nan
    assert np.isnan(oracle.fdrstats(M2)[1])


def test_fdrdenormalize_promotion(oracle):
    m, s = np.float32(1.2345678), np.float32(0.7654321)
    t32 = oracle.fdrdenormalize(10, m, s)
    assert isinstance(t32, np.float32)
    assert t32 == np.float32(np.float32(np.float32(10) * s) + m)
    t64 = oracle.fdrdenormalize(10.0, m, s)
    assert isinstance(t64, float) and t64 == 10.0 * float(s) + float(m)
    # a Float32 element one ulp below the Float32 threshold is not a proto-hit, at it is
    x = np.array([[np.nextafter(t32, np.float32(-np.inf))], [t32]], dtype=np.float32)
    assert oracle.findprotohits(x, t32).tolist() == [[1, 0]]
