"""GPU tests of the HDF5 filterbank ingest: the device bit transpose (fdr_bitunshuffle)
against the oracle, spectrograms read from rawspec-style bitshuffle+LZ4 HDF5 files equal to
the data written, the heavytests.jl stand-in (test/heavytests.jl:11-39: channels
659935:660084 of IF 1, rates 0:-0.25:-5, peak at CartesianIndex(55, 11)) read through an
HDF5 file, and the multi-channel search of an HDF5 file equal to that of the same data as a
filterbank file."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("es,nelem,block", [(4, 8192, 2048), (4, 1005, 256), (4, 7, 8), (1, 4099, 128),
                                            (2, 333, 64), (8, 2000, 512)])
def test_bitunshuffle_matches_oracle(fdr, oracle, es, nelem, block):
    rng = np.random.default_rng(nelem + es)
    raw = rng.integers(0, 256, nelem * es, dtype=np.uint8).tobytes()
    whole = nelem - nelem % 8
    sh = b"".join(oracle.bitshuffle_block(raw[e * es:min(whole, e + block) * es], es)
                  for e in range(0, whole, block)) + raw[whole * es:]
    d_in = torch.tensor(np.frombuffer(sh, np.uint8), device="cuda")
    d_out = torch.empty(nelem * es, dtype=torch.uint8, device="cuda")
    lib = fdr._lib.lib()
    fdr._lib.check(lib.fdr_bitunshuffle(d_in.data_ptr(), nelem, es, block, d_out.data_ptr(), None))
    assert d_out.cpu().numpy().tobytes() == raw
    assert lib.fdr_bitunshuffle(d_in.data_ptr(), nelem, 3, block, d_out.data_ptr(), None) == \
        fdr._lib.FDR_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("shape,chunk,ranges", [
    ((16, 1, 70000), (16, 1, 1 << 14), [(0, 70000), (16000, 17000), (65530, 70000)]),
    ((9, 2, 5000), (4, 1, 1024), [(3, 4999), (0, 1)]),
])
def test_h5_spectrogram_equals_data(fdr, tmp_path, shape, chunk, ranges):
    rng = np.random.default_rng(shape[2])
    data = rng.exponential(1.0, shape).astype(np.float32)
    path = str(tmp_path / "d.h5")
    fdr.write_fbh5(path, {"fch1": 1.0, "foff": 1.0, "tsamp": 1.0}, data, chunk=chunk)
    fb = fdr.H5Filterbank(path)
    assert (fb.nsamples, fb.nifs, fb.nchans) == shape
    for ifno in range(shape[1]):
        for lo, hi in ranges:
            got = fb.spectrogram(lo, hi, ifno)
            assert got.shape == (hi - lo, shape[0]) and got.stride() == (1, hi - lo)
            assert np.array_equal(got.cpu().numpy(), data[:, ifno, lo:hi].T)
        got = fb.spectrogram(10, 900, ifno, t0=2, nt=3)
        assert np.array_equal(got.cpu().numpy(), data[2:5, ifno, 10:900].T)


def test_heavytest_standin_through_hdf5(fdr, tmp_path):
    """A drifting tone at channel 659935 + 54 (zero-based), -2.5 ch/step, in a 2^20-channel
    rawspec-style file; the reference's slice h5["data"][659935 .+ (0:149), 1, :] and rates
    0:-0.25:-5 put the peak of intfdr, fftfdr and zdtfdr at zero-based (54, 10)."""
    Nf, Nt = 1 << 20, 16
    rng = np.random.Generator(np.random.PCG64(11))
    data = rng.exponential(1.0, size=(Nt, 1, Nf)).astype(np.float32)
    base = 659935
    for t in range(Nt):
        c = base + 54 - 2.5 * t
        lo = int(np.floor(c))
        f = c - lo
        data[t, 0, lo] += 40 * (1 - f)
        data[t, 0, lo + 1] += 40 * f
    path = str(tmp_path / "voyager_standin.h5")
    fdr.write_fbh5(path, {"fch1": 8421.38671875, "foff": -2.7939677238464355e-06, "tsamp": 18.253611008,
                          "nbits": 32, "source_name": "VOYAGER-1"}, data)
    fb = fdr.H5Filterbank(path)
    spec = fb.spectrogram(base, base + 150)
    rates = [0.0 - 0.25 * j for j in range(21)]
    outs = [fdr.intfdr(spec, rates), fdr.fftfdr(fdr.fftfdr_workspace(spec), rates),
            fdr.zdtfdr(fdr.ZDTWorkspace(spec, 0.0, -0.25, 21))]
    for out in outs:
        a = out.cpu().numpy()
        assert np.unravel_index(np.argmax(a), a.shape) == (54, 10)


def test_pipeline_on_hdf5_matches_filterbank(fdr, oracle, tmp_path):
    nfpc, nt, nco = 1 << 14, 16, 3
    data = np.empty((nt, 1, nfpc * nco), np.float32)
    for c in range(nco):
        spec, _ = oracle.synth_spectrogram(nfpc, nt, 2, 20.0, 40.0, 3.5, seed=300 + c)
        data[:, 0, c * nfpc:(c + 1) * nfpc] = spec.T
    hdr = {"fch1": 8000.0, "foff": -2.8e-6, "tsamp": 18.25, "nbits": 32, "source_name": "SYNTH"}
    fil, h5 = str(tmp_path / "s.fil"), str(tmp_path / "s.h5")
    fdr.write_filterbank(fil, hdr, data)
    fdr.write_fbh5(h5, hdr, data, chunk=(nt, 1, 5000))  # chunks straddle coarse channels
    pipe = fdr.SearchPipeline(nfpc, nt, -4.0, 0.125, 65, snr=10.0)
    a = pipe.run(fdr.Filterbank(fil))
    b = pipe.run(fdr.H5Filterbank(h5))
    assert [r[0] for r in a] == [r[0] for r in b]
    for ra, rb in zip(a, b):
        assert np.array_equal(ra[1], rb[1]) and np.array_equal(ra[2], rb[2])
        assert ra[3].tobytes() == rb[3].tobytes()
