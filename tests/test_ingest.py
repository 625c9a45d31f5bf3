"""Filterbank ingest (host side): header and data round trip, the coarse-channel spectrogram
layout, and malformed files."""
import numpy as np
import pytest


def _hdr():
    return {"telescope_id": 6, "machine_id": 10, "data_type": 1, "source_name": "SYNTH",
            "rawdatafile": "synth.raw", "tstart": 59046.9, "tsamp": 18.253611008,
            "fch1": 8421.38671875, "foff": -2.7939677238464355e-06, "nbits": 32, "nifs": 1,
            "az_start": 0.0, "za_start": 0.0, "src_raj": 171010.0, "src_dej": 121944.0}


def test_roundtrip_and_layout(fdr, tmp_path):
    rng = np.random.default_rng(0)
    data = rng.random((16, 1, 96), dtype=np.float32)  # (time, IF, channel)
    path = str(tmp_path / "a.fil")
    fdr.write_filterbank(path, _hdr(), data)
    fb = fdr.Filterbank(path)
    for k, v in _hdr().items():
        assert fb.header[k] == v
    assert fb.nsamples == 16 and fb.nchans == 96
    assert np.array_equal(np.asarray(fb.data), data)
    spec = fb.spectrogram(32, 64)
    assert spec.shape == (32, 16)
    assert np.array_equal(spec, data[:, 0, 32:64].T)
    assert spec.strides == (4, 32 * 4)  # frequency fastest, as a Julia matrix
    part = fb.spectrogram(0, 8, t0=4, nt=8)
    assert np.array_equal(part, data[4:12, 0, 0:8].T)


def test_8bit_and_two_ifs(fdr, tmp_path):
    rng = np.random.default_rng(1)
    data = rng.integers(0, 255, (8, 2, 40)).astype(np.uint8)
    hdr = _hdr()
    hdr["nbits"] = 8
    path = str(tmp_path / "b.fil")
    fdr.write_filterbank(path, hdr, data)
    fb = fdr.Filterbank(path)
    spec = fb.spectrogram(10, 20, ifno=1)
    assert spec.dtype == np.float32
    assert np.array_equal(spec, data[:, 1, 10:20].T.astype(np.float32))


def test_malformed(fdr, tmp_path):
    path = str(tmp_path / "c.fil")
    with open(path, "wb") as fh:
        fh.write(b"\x05\x00\x00\x00HELLO")
    with pytest.raises(ValueError):
        fdr.Filterbank(path)
    with pytest.raises(ValueError):
        fdr.write_filterbank(str(tmp_path / "d.fil"), {"bogus_key": 1}, np.zeros((2, 4), np.float32))
