"""GPU tests of the batched multi-channel ZDT (fdr_batch_*): uneven shapes, shared plans,
staged channels, autotuning and CUDA-graph replay, against per-channel zdtfdr and the FP64
oracle (relative L-infinity 1e-5; per-channel results are bit-identical to single zdtfdr!
calls because the same kernels run)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _channels(oracle):
    shapes = [(2 ** 14, 16, -2.0, 1 / 16, 65), (2 ** 15, 32, -4.0, 1 / 16, 129),
              (2 ** 14, 64, -2.0, 1 / 16, 65), (3000, 16, -1.0, 0.25, 9),
              (2 ** 14, 16, -8.0, 1 / 16, 257), (2 ** 14, 16, 0.5, 1 / 16, 65)]
    out = []
    for i, (Nf, Nt, r0, dr, Nr) in enumerate(shapes):
        spec, _ = oracle.synth_spectrogram(Nf, Nt, 3, 8, 50, 4, seed=100 + i)
        out.append((spec, r0, dr, Nr))
    return out


def test_batch_matches_single_calls(fdr, oracle):
    ch = _channels(oracle)
    b = fdr.ZDTBatch(ch, slots=2)
    info = b.info()
    assert info["channels"] == len(ch) and info["fused"] == len(ch) - 1
    outs = [o.cpu().numpy() for o in b.launch()]
    for (spec, r0, dr, Nr), o in zip(ch, outs):
        single = fdr.zdtfdr(fdr.ZDTWorkspace(spec, r0, dr, Nr)).cpu().numpy()
        np.testing.assert_array_equal(o, single)
    for idx in (0, 3):
        spec, r0, dr, Nr = ch[idx]
        truth = oracle.fdr_truth(spec, [r0 + dr * j for j in range(Nr)][::8])
        assert oracle.rel_linf(outs[idx][:, ::8], truth) < 1e-5


def test_batch_autotune_capture_replay(fdr, oracle):
    ch = _channels(oracle)
    b = fdr.ZDTBatch(ch, slots=4)
    eager = [o.cpu().numpy() for o in b.launch()]
    tun = b.autotune()
    assert tun["active_slots"] in (1, 2, 4)
    assert len(tun["groups_per_shape"]) == 4 and all(g >= 1 for g in tun["groups_per_shape"])
    s = torch.cuda.Stream()
    b.capture(stream=s)
    assert b.info()["captured"]
    for o in b.outputs:
        o.zero_()
    for _ in range(2):
        b.launch(stream=s)
    s.synchronize()
    for e, o in zip(eager, b.outputs):
        np.testing.assert_array_equal(e, o.cpu().numpy())
