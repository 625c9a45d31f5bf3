"""Multi-coarse-channel search from a filterbank file: the double-buffered pipeline finds
the same proto-hits as searching each coarse channel directly, and its clusters sit at the
injected tones."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pipeline_matches_direct_search(fdr, oracle, tmp_path):
    nfpc, nt, nco = 1 << 14, 16, 4
    rng = np.random.default_rng(5)
    data = np.empty((nt, 1, nfpc * nco), np.float32)
    tones = []
    for c in range(nco):
        spec, tl = oracle.synth_spectrogram(nfpc, nt, 2, 20.0, 40.0, 3.5, seed=100 + c)
        data[:, 0, c * nfpc:(c + 1) * nfpc] = spec.T
        tones.append(tl)
    hdr = {"fch1": 8000.0, "foff": -2.8e-6, "tsamp": 18.25, "nbits": 32, "source_name": "SYNTH"}
    path = str(tmp_path / "s.fil")
    fdr.write_filterbank(path, hdr, data)
    fb = fdr.Filterbank(path)
    pipe = fdr.SearchPipeline(nfpc, nt, -4.0, 0.125, 65, snr=10.0)
    res = pipe.run(fb)
    assert [r[0] for r in res] == list(range(nco))
    ws = fdr.ZDTWorkspace(None, -4.0, 0.125, 65, shape=(nfpc, nt))
    dest = fdr.fortran_empty(nfpc, 65)
    for c, hits, labels, clusters in res:
        spec = fdr.as_device_f32(data[:, 0, c * nfpc:(c + 1) * nfpc].T)
        ref = fdr.zdtfdr_protohits_(dest, ws, spec, threshold=10.0, snr=True)
        assert np.array_equal(hits, ref)
        assert clusters["count"].sum() == len(hits)
        for c0, r, a in tones[c]:  # every injected tone peaks in some cluster near (c0, r)
            near = [k for k in clusters
                    if abs(((int(k["peak_i"]) - c0 + nfpc / 2) % nfpc) - nfpc / 2) <= 2
                    and abs(-4.0 + 0.125 * int(k["peak_j"]) - r) <= 0.25]
            assert near, (c, c0, r)
    # a second run over the same pipeline (buffers reused) gives the same result
    res2 = pipe.run(fb, channels=[2, 0])
    assert np.array_equal(res2[0][1], res[2][1]) and np.array_equal(res2[1][1], res[0][1])
    rows = pipe.hit_table(fb, res)
    assert rows and all(abs(r["freq"] - (8000.0 - 2.8e-6 * r["channel"])) < 1e-9 for r in rows)
