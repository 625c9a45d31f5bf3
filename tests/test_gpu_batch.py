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


def test_batch_config4_shapes(fdr, oracle):
    """Channels drawn from the batched workload's own sets -- Nf in {2^18, 2^19, 2^20}, Nt in
    {16, 32, 64}, drift spans +-2/+-4/+-8 ch/step at step 1/16 (65, 129 or 257 rates) -- in
    one captured batch: every channel bit-identical to its single zdtfdr! call and sampled
    columns within 1e-5 of the FP64 truth."""
    rng = np.random.default_rng(44)
    combos = [(1 << 18, 64, 8), (1 << 19, 32, 4), (1 << 20, 16, 2), (1 << 20, 64, 2),
              (1 << 18, 16, 8), (1 << 19, 64, 4)]
    ch = []
    for i, (Nf, Nt, span) in enumerate(combos):
        spec, _ = oracle.synth_spectrogram(Nf, Nt, int(rng.integers(0, 11)), 8, 50, span, seed=400 + i)
        ch.append((spec, -float(span), 1 / 16, 2 * span * 16 + 1))
    b = fdr.ZDTBatch(ch, slots=4)
    b.autotune()
    s = torch.cuda.Stream()
    b.capture(stream=s)
    b.launch(stream=s)
    s.synchronize()
    for (spec, r0, dr, Nr), o in zip(ch, b.outputs):
        got = o.cpu().numpy()
        single = fdr.zdtfdr(fdr.ZDTWorkspace(spec, r0, dr, Nr)).cpu().numpy()
        np.testing.assert_array_equal(got, single)
        cols = [0, Nr // 3, Nr - 1]
        truth = oracle.fdr_truth(spec, [r0 + dr * j for j in cols])
        assert oracle.rel_linf(got[:, cols], truth) < 1e-5
