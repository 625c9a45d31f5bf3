"""Taylor-tree integer FDR (fdr_taylor_tree): bit-exact with the float32 restatement of the
same additions in the oracle, and equal to intfdr along the tree paths (integer-valued data,
so that every summation order is exact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("Nf,Nt,dmin,dmax", [
    (4096, 16, -15, 15), (3000, 16, -4, 9), (1000, 2, -1, 1), (513, 4, 0, 3),
    (20, 16, -15, 15),  # fewer channels than the halo: the paths wrap several times
    (1 << 16, 32, -31, 31), (5000, 64, -63, 63), (1 << 20, 16, -15, 15)])
def test_taylor_matches_oracle(fdr, oracle, Nf, Nt, dmin, dmax):
    rng = np.random.default_rng(Nf + Nt)
    spec = (-np.log(rng.random((Nf, Nt)))).astype(np.float32)
    out = fdr.taylorfdr(spec, dmin, dmax).cpu().numpy()
    assert np.array_equal(out, oracle.taylor_tree(spec, dmin, dmax))


def test_taylor_paths_and_intfdr(fdr, oracle):
    rng = np.random.default_rng(3)
    Nf, Nt = 2048, 16
    spec = rng.integers(0, 100, (Nf, Nt)).astype(np.float32)  # exact in any order
    out = fdr.taylorfdr(spec).cpu().numpy()
    drifts = list(range(-(Nt - 1), Nt))
    shifts = np.array([fdr.taylor_shifts(Nt, d) for d in drifts], dtype=np.int64)
    # intfdr along the tree paths (caller-given shifts)
    import ctypes as C
    dspec = fdr.as_device_f32(spec)
    dst = fdr.fortran_empty(Nf, len(drifts))
    arr = (C.c_int64 * shifts.size)(*shifts.ravel().tolist())
    fdr._lib.check(fdr._lib.lib().fdr_intfdr_shifts(fdr.arrays.ptr(dspec), Nf, Nt, arr, len(drifts),
                                                    fdr.arrays.ptr(dst), fdr.arrays.stream_handle()))
    assert np.array_equal(out, dst.cpu().numpy())
    # straight lines: d = 0, +-(Nt-1) are intfdr at rates 0, +-1
    lines = fdr.intfdr(spec, [-1.0, 0.0, 1.0]).cpu().numpy()
    assert np.array_equal(out[:, [0, Nt - 1, 2 * Nt - 2]], lines)


def test_taylor_argument_errors(fdr):
    spec = np.ones((64, 12), np.float32)
    with pytest.raises(fdr.FDRError):
        fdr.taylorfdr(spec)  # Nt not a power of two
    with pytest.raises(fdr.FDRError):
        fdr.taylorfdr(np.ones((64, 8), np.float32), -8, 0)
