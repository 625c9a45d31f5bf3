"""GPU tests of intshift/intfdr (intfdr.jl): bit-exact with the oracle's restatement of
the reference's CPU algorithm (sequential float32 sum in time order)."""
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_known_answers(fdr, golden):
    d = np.array(golden["spectrogram"], dtype=np.float32)
    sh = fdr.intshift(d, golden["intshift_rate"]).cpu().numpy()
    assert np.array_equal(sh, np.array(golden["intshift_expected"], dtype=np.float32))
    out = fdr.intfdr(d, golden["rates"]).cpu().numpy()
    assert np.array_equal(out, np.array(golden["fdr_expected"], dtype=np.float32))


@pytest.mark.parametrize("Nf,Nt", [(65536, 16), (1000, 7), (3, 2), (1, 1), (4097, 33)])
def test_bit_exact_fractional_rates(fdr, oracle, Nf, Nt):
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 20, 20, 4, seed=Nf + Nt)
    rates = [-4.0 + 0.25 * j for j in range(33)]  # many ties at x.5 -> ties to even
    out = fdr.intfdr(spec, rates).cpu().numpy()
    ref = oracle.intfdr(spec, rates)
    assert np.array_equal(bits(out), bits(ref))


def test_bit_exact_float32_and_rational_rates(fdr, oracle):
    spec, _ = oracle.synth_spectrogram(8192, 16, 3, 20, 20, 4, seed=77)
    r32 = (np.arange(-30, 31, dtype=np.float32) * np.float32(0.1)).astype(np.float32)
    out = fdr.intfdr(spec, r32).cpu().numpy()
    ref = oracle.intfdr(spec, list(r32), rate_dtype="f32")
    assert np.array_equal(bits(out), bits(ref))
    rb = fdr.batchrates(16, 1.0, -4.0, Nrb=360)[0]
    rl = list(rb)
    assert all(isinstance(r, Fraction) for r in rl)
    out = fdr.intfdr(spec, rl).cpu().numpy()
    ref = oracle.intfdr(spec, rl, rate_dtype="rational")
    assert np.array_equal(bits(out), bits(ref))


def test_bit_exact_config2_size(fdr, oracle):
    """Nf=2^20, Nt=16, rates -4:1/16:4 (129 rates)."""
    spec, _ = oracle.synth_spectrogram(2 ** 20, 16, 20, 8, 50, 4, seed=2000)
    rates = [-4.0 + j / 16 for j in range(129)]
    out = fdr.intfdr(spec, rates).cpu().numpy()
    idx = [0, 17, 64, 100, 128]
    ref = oracle.intfdr(spec, [rates[i] for i in idx])
    assert np.array_equal(bits(out[:, idx]), bits(ref))


def test_large_shifts_wrap(fdr, oracle):
    spec, _ = oracle.synth_spectrogram(1024, 8, 2, 20, 20, 4, seed=3)
    rates = [-5000.5, -1024.0, 1023.0, 3.5e6]
    out = fdr.intfdr(spec, rates).cpu().numpy()
    ref = oracle.intfdr(spec, rates)
    assert np.array_equal(bits(out), bits(ref))


@pytest.mark.parametrize("Nf,Nt,rates", [
    (4096, 16, [float(r) for r in range(-15, 16)]),   # shared-memory windows, wrapping at 0
    (1024, 16, [float(r) for r in range(-15, 16)]),   # spread > Nf/4: per-element kernel
    (8192, 80, [-2.0, -0.5, 0.25, 1.5]),              # Nt > 64: per-element kernel
    (777, 9, [-1.5, 0.5, 2.5]),                       # ragged last tile
])
def test_bit_exact_tiled_and_untiled(fdr, oracle, Nf, Nt, rates):
    """Both intfdr kernels (shared-memory windows where every rate's shift of a time step
    lies within Nf/4 of the others, per-element gathers otherwise) give the reference's
    float32 sums bit for bit."""
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 20, 20, 4, seed=Nf + 3 * Nt)
    out = fdr.intfdr(spec, rates).cpu().numpy()
    ref = oracle.intfdr(spec, rates)
    assert np.array_equal(bits(out), bits(ref))


def test_intshift_random(fdr, oracle):
    spec, _ = oracle.synth_spectrogram(4096, 16, 2, 20, 20, 4, seed=4)
    for r in [-3.75, 0.5, 2.25, 17.0]:
        assert np.array_equal(fdr.intshift(spec, r).cpu().numpy(), oracle.intshift(spec, r))


def test_intfdr_inplace_and_errors(fdr, oracle):
    spec, _ = oracle.synth_spectrogram(512, 4, 1, 20, 20, 2, seed=5)
    dest = fdr.fortran_empty(512, 3)
    fdr.intfdr_(dest, spec, [-1.0, 0.0, 1.0])
    assert np.array_equal(dest.cpu().numpy(), oracle.intfdr(spec, [-1.0, 0.0, 1.0]))
    with pytest.raises(fdr.FDRError):
        fdr.intfdr_(fdr.fortran_empty(512, 2), spec, [-1.0, 0.0, 1.0])
