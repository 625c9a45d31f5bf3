"""Proto-hit clustering (fdr_cluster_protohits) against the union-find restatement in the
oracle: labels and every cluster summary must match exactly."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _random_hits(rng, Nf, Nj, density):
    mask = rng.random((Nj, Nf)) < density       # [j][i]
    j, i = np.nonzero(mask)                      # ordered by (j, i) = column-major order
    return np.stack([i, j], axis=1).astype(np.int64)


def _compare(fdr, oracle, hits, Nf, Nj, di, dj, mats):
    labels, cl = fdr.cluster_protohits(hits, Nf, Nj, di, dj, fdr=mats)
    host = None
    if mats is not None:
        host = [m.cpu().numpy() for m in (mats if isinstance(mats, list) else [mats])]
    rl, rc = oracle.cluster_protohits(hits, Nf, di, dj, fdr=host)
    assert np.array_equal(labels, rl)
    assert len(cl) == len(rc)
    for a, b in zip(cl, rc):
        for k in ("count", "i_min", "i_max", "j_min", "j_max", "first", "peak_i", "peak_j"):
            assert int(a[k]) == b[k], (k, a, b)
        if mats is None:
            assert np.isnan(a["peak_value"])
        else:
            assert np.float32(a["peak_value"]) == np.float32(b["peak_value"])


@pytest.mark.parametrize("di,dj", [(1, 1), (0, 1), (2, 3), (1, 0), (0, 0)])
def test_random_hits_match_oracle(fdr, oracle, di, dj):
    rng = np.random.default_rng(100 + 10 * di + dj)
    Nf, Nj = 96, 40
    hits = _random_hits(rng, Nf, Nj, 0.22)
    vals = rng.integers(0, 5, (Nf, Nj)).astype(np.float32)  # many ties
    mats = fdr.as_device_f32(vals)
    _compare(fdr, oracle, hits, Nf, Nj, di, dj, mats)
    _compare(fdr, oracle, hits, Nf, Nj, di, dj, None)


def test_rate_batches_and_edges(fdr, oracle):
    rng = np.random.default_rng(7)
    Nf, Nrb = 50, 12
    hits = _random_hits(rng, Nf, 2 * Nrb, 0.3)
    # proto-hits on the first and last channel: no wrap-around
    hits = np.unique(np.concatenate([hits, [[0, 3], [Nf - 1, 3]]]), axis=0)
    hits = hits[np.lexsort((hits[:, 0], hits[:, 1]))]
    vals = rng.standard_normal((Nf, 2 * Nrb)).astype(np.float32)
    mats = [fdr.as_device_f32(vals[:, :Nrb]), fdr.as_device_f32(vals[:, Nrb:])]
    _compare(fdr, oracle, hits, Nf, 2 * Nrb, 1, 1, mats)


def test_clusters_of_a_zdt(fdr, oracle):
    spec, tones = oracle.synth_spectrogram(1 << 14, 16, 6, 15.0, 40.0, 4.0, seed=21)
    ws = fdr.ZDTWorkspace(spec, -4.0, 0.125, 65)
    out = fdr.zdtfdr(ws)
    hits = fdr.findprotohits(out, 8.0, snr=True)
    assert len(hits) > 0
    _compare(fdr, oracle, hits, 1 << 14, 65, 1, 1, out)
    labels, cl = fdr.cluster_protohits(hits, 1 << 14, 65, 1, 1, fdr=out)
    assert cl["count"].sum() == len(hits)
    assert len(cl) < len(hits)  # proto-hits of one signal merge


def test_empty_errors_and_capacity(fdr):
    labels, cl = fdr.cluster_protohits(np.zeros((0, 2), np.int64), 10, 10)
    assert len(labels) == 0 and len(cl) == 0
    with pytest.raises(fdr.FDRError):  # not in column-major order
        fdr.cluster_protohits(np.array([[3, 1], [2, 1]]), 10, 10)
    with pytest.raises(fdr.FDRError):  # repeated proto-hit
        fdr.cluster_protohits(np.array([[2, 1], [2, 1]]), 10, 10)
    with pytest.raises(fdr.FDRError):  # out of range
        fdr.cluster_protohits(np.array([[2, 1], [12, 1]]), 10, 10)
    hits = np.array([[0, 0], [5, 0], [9, 9]])
    with pytest.raises(fdr.CapacityError):
        fdr.cluster_protohits(hits, 10, 10, capacity=2)
    labels, cl = fdr.cluster_protohits(torch.from_numpy(hits).cuda(), 10, 10)
    assert list(labels) == [0, 1, 2] and list(cl["count"]) == [1, 1, 1]
