"""CPU tests of the C-ABI library and the host-side logic (no kernels launched)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fdr_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdr_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol(fdr):
    lib = fdr._lib.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared entry point has a ctypes signature in the binding
    assert set(names) <= set(fdr._lib.SIGNATURES), set(names) - set(fdr._lib.SIGNATURES)


def test_version_and_status_strings(fdr):
    lib = fdr._lib.lib()
    assert b"sm_100a" in lib.fdr_version()
    assert lib.fdr_status_string(0) == b"FDR_OK"
    assert lib.fdr_status_string(6) == b"FDR_ERR_CAPACITY"


def test_zdtutils_via_abi(fdr, oracle):
    for Nt, Nr in [(16, 129), (16, 33), (2, 3), (64, 257), (32, 65), (16, 1)]:
        assert fdr.calcNl(Nt, Nr) == oracle.calcNl(Nt, Nr)
        assert fdr.growNr(Nt, Nr) == oracle.growNr(Nt, Nr)
    assert fdr.calcNl(16, 129, (2,)) == 256
    assert fdr.calcNl(16, 129, (2, 3, 5, 7)) == oracle.calcNl(16, 129, (2, 3, 5, 7))
    assert fdr.estimate_memory(2 ** 20, 16, 129, 2, 3) == oracle.estimate_memory(2 ** 20, 16, 129, 2, 3)
    with pytest.raises(ValueError):
        fdr.calcNl(16, 129, (1,))


def test_argument_errors_without_device(fdr):
    lib = fdr._lib.lib()
    h = C.c_void_p()
    st = lib.fdr_zdt_create(C.byref(h), None, 0, 16, 0.0, 1.0, 10, None, 0, 0, None)
    assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT
    assert b"bad sizes" in lib.fdr_last_error_string()
    st = lib.fdr_zdt_create(C.byref(h), None, 67 * 2, 16, 0.0, 1.0, 10, None, 0, 0, None)
    assert st == fdr._lib.FDR_ERR_UNSUPPORTED_SIZE
    st = lib.fdr_intfdr(None, 10, 2, None, 1, 0, None, None)
    assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT
    cnt = C.c_int64()
    st = lib.fdr_findprotohits(None, 1, 10, 2, 1.0, 0, None, 0, C.byref(cnt), None, None)
    assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT


def test_fused_split_plan(fdr):
    """The four-step split of the fused path, chosen on the host: 512 bins per czt CTA up to
    Nf = 2^20 with F in registers (Nt <= 16), 1024 above (mixed-precision workspaces split
    the same way: their tensor-core output passes cover P = 1024 and 2048), 512 / 256 bins with F
    in shared memory (Nt <= 32 / 64), and 512 bins at Nf = 2^20 and 2^21 for 32 < Nt <= 64
    (F split over a two-CTA cluster); the staged kernels outside 2^12..2^22 or P > 4096."""
    fs = fdr.fused_split
    assert fs(2 ** 20, 16, 129) == (2048, 512)
    assert fs(2 ** 20, 16, 129, mixed_precision=True) == (2048, 512)
    assert fs(2 ** 19, 16, 129, mixed_precision=True) == (1024, 512)
    assert fs(2 ** 19, 16, 129) == (1024, 512)
    assert fs(2 ** 21, 16, 17) == (2048, 1024)
    assert fs(2 ** 22, 16, 17) == (4096, 1024)
    assert fs(2 ** 20, 24, 33) == (2048, 512)
    assert fs(2 ** 20, 64, 65) == (2048, 512)
    assert fs(2 ** 21, 33, 9) == (4096, 512)
    assert fs(2 ** 19, 64, 65) == (2048, 256)
    assert fs(2 ** 18, 40, 33) == (1024, 256)
    assert fs(2 ** 12, 16, 17) == (64, 64)
    for Nf, Nt in ((2 ** 23, 16), (2 ** 11, 16), (3 * 2 ** 18, 16), (2 ** 20, 65), (2 ** 22, 64)):
        assert fs(Nf, Nt, 17) is None, (Nf, Nt)
    assert fs(2 ** 20, 16, 129, staged_only=True) is None
    for Nf, Nt in ((2 ** 16, 16), (2 ** 20, 16), (2 ** 21, 32)):
        P, Q = fs(Nf, Nt, 33)
        assert P * Q == Nf


def test_batchrates_host_matches_oracle(fdr, oracle):
    for args in [(16, 1.0, -4.0, None, 360), (16, 0.5, 10.0, -3.0, 50),
                 (32, -0.25, -2.0, 5.0, 40), (17, 0.1, -100.0, 100.0, 360), (64, 1.0, -8.0, 8.0, 100)]:
        Nt, dh, r1, r2, Nrb = args
        mine = fdr.batchrates(Nt, dh, r1, r2, Nrb=Nrb)
        ref = oracle.batchrates(Nt, dh, r1, r2, Nrb=Nrb)
        assert [list(b) for b in mine] == ref


# Expected batches worked by hand from src/batchrates.jl:22-60 (not from a transcription):
# nc = round(r / δ) ties to even; Nrspan = |nc2 - nc1| + 1; Nrb = growNr(Nt, min(Nrb, Nrspan))
# = nextprod((2,3,5), Nt + Nrb - 1) - Nt + 1; Nr = cld(Nrspan, Nrb) * Nrb; the bonus
# Nr - Nrspan goes sign(δ)*bonus/2 rounded from zero below nc1 and rounded to zero above
# nc2; rates nc1//(Nt-1) .. nc2//(Nt-1) in Nr equal steps, Nrb per batch.
#   (args, Nrb kw) -> [(first, step, length) per batch]
HAND_BATCHES = [
    # span -4..4 Hz/s at 1 Hz/s, Nt=16: nc -4..4, Nrspan 9, 16+9-1 = 24 is smooth: Nrb 9, no bonus
    ((16, 1.0, -4.0, None), 360, [("-4/15", "1/15", 9)]),
    # 0..21: Nrspan 22, 16+22-1 = 37 -> 40, Nrb 25, bonus 3 (odd): 2 below (from zero), 1 above
    ((16, 1.0, 0.0, 21.0), 360, [("-2/15", "1/15", 25)]),
    # the same span with δ < 0: nc1 = round(-0.0) = 0, nc2 = -21; sign -1: -1.5 from zero = -2,
    # so nc1 = 0 + 2 = 2; -1.5 to zero = -1, so nc2 = -22; the rates descend
    ((16, -1.0, 0.0, 21.0), 360, [("2/15", "-1/15", 25)]),
    # -100..100 with Nrb 50: Nrspan 201, 16+50-1 = 65 -> 72, Nrb 57, Nr = cld(201,57)*57 = 228,
    # bonus 27: 14 below (13.5 from zero), 13 above (13.5 to zero): -114..113 over 15
    ((16, 1.0, -100.0, 100.0), 50, [("-114/15", "1/15", 57), ("-57/15", "1/15", 57),
                                    ("0", "1/15", 57), ("57/15", "1/15", 57)]),
    # r1 > r2 swaps; Nt=32, δ 2 Hz/s: nc -5..5, Nrspan 11, 32+11-1 = 42 -> 45, Nrb 14, bonus 3
    ((32, 2.0, 10.0, -10.0), 360, [("-7/31", "1/31", 14)]),
    # ties to even: 2.5 -> 2, 7.5 -> 8; Nrspan 7, 16+7-1 = 22 -> 24, Nrb 9, bonus 2: 1 and 1
    ((16, 1.0, 2.5, 7.5), 360, [("1/15", "1/15", 9)]),
]


@pytest.mark.parametrize("args,nrb,expected", HAND_BATCHES)
def test_batchrates_hand_derived(fdr, args, nrb, expected):
    from fractions import Fraction
    got = fdr.batchrates(*args, Nrb=nrb)
    assert [(b.first, b.step, len(b)) for b in got] == \
        [(Fraction(a), Fraction(s), n) for a, s, n in expected]


def test_rate_range_params(fdr):
    rr = fdr.batchrates(16, 1.0, -4.0)[0]
    assert rr.first == rr.start and len(rr) == rr.length
    assert list(rr)[1] - list(rr)[0] == rr.step


def test_proposal_calibration_host_logic(fdr):
    """Threshold calibration of the proposal search (host code, no GPU)."""
    import numpy as np
    P = fdr.proposal
    rng = np.random.default_rng(0)
    counts = np.zeros((50, 16), np.int64)
    probs = np.full((50, 16), 0.001)
    for i in range(50):
        w = rng.choice(16, 2, replace=False)
        counts[i, w] = rng.integers(1, 20, 2)
        probs[i, w] = rng.uniform(0.3, 0.99, 2)
    cal = P.calibrate(probs, counts, target=1.0)
    assert cal["window_recall"] == 1.0 and cal["fallback_rate"] == 0.0
    assert cal["cost"] == 100.0  # exactly the two positive windows per channel
    # hide one positive window below every other probability: recall 1.0 needs fallback
    probs[0, np.nonzero(counts[0])[0][0]] = 0.0005
    cal = P.calibrate(probs, counts, target=1.0)
    assert cal["window_recall"] == 1.0 and cal["cost"] > 100.0
