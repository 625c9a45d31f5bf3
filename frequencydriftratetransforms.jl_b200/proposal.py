"""Learned drift-rate window proposal (fdr_propose_* in the C ABI).

The reference has no learned component; this is a serving extension of its batched-rate
search (batchrates.jl:22-60, the r0 iterator of zdtfdr!, zdtfdr.jl:354).  For a coarse
channel (Nf x Nt spectrogram) a small 1-D conv net reads a downsampled view of the channel
and predicts which of 16 drift-rate windows (1 ch/step wide, [-8, 8) ch/step at step 1/16,
16 rates each) hold proto-hits.  ``ProposalSearch`` then runs zdtfdr! + findprotohits only
over the proposed windows and falls back to the full 256-rate search when the network is
not confident.

Two network inputs (``lag``):

* ``lag=False``: the 256-channel sum-downsampled power, Nt x Nf/256 (features()).
* ``lag=True``: the same plus 17 rows of per-bin adjacent-step lag products for lags -8..8
  (fdr_propose_lag_features), which carry the drift rate that a 256-channel bin hides
  (a tone drifting <= 8 ch/step moves less than one bin over 16 steps).

Training data: seeded synthetic channels labelled by full plain ZDT + findprotohits
(``FullSearch``, ``make_batch``); the network is trained online by the library's own
forward/backward/Adam kernels (``train_online``).  Checkpoints are a flat binary file with
a JSON header (weights, Adam moments, step), so training resumes bit for bit.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import struct
import time

import numpy as np
import torch

from . import _lib
from .arrays import fortran_empty, ptr, stream_handle
from .zdt import ZDTWorkspace, zdtfdr_blocks_protohits_, zdtfdr_protohits_

NWIN, RATES_PER_WIN = 16, 16
DR = 1.0 / 16
R_MIN = -8.0
NRATES = NWIN * RATES_PER_WIN
FACTOR = 256
MAXLAG = 8


def input_channels(Nt, lag):
    return Nt + (2 * MAXLAG + 1 if lag else 0)


class ProposalNet:
    """Handle on a device-resident network (fdr_propose_create)."""

    def __init__(self, nbins=4096, cin=16, max_batch=64, seed=1, lag=False, compress=True):
        h = C.c_void_p()
        _lib.check(_lib.lib().fdr_propose_create(C.byref(h), nbins, cin, 32, 5, NWIN, max_batch,
                                                 C.c_uint64(seed)))
        self._h = h
        self.nbins, self.cin, self.max_batch, self.seed = nbins, cin, max_batch, seed
        self.lag, self.compress = lag, compress
        self.meta = {}
        n = C.c_int64()
        _lib.check(_lib.lib().fdr_propose_num_params(self._h, C.byref(n)))
        self.nparams = n.value
        self._logits = torch.empty((max_batch, NWIN), dtype=torch.float32, device="cuda")
        self._loss = torch.empty(1, dtype=torch.float32, device="cuda")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().fdr_propose_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, x):
        """x: (B, cin, nbins) float32 CUDA tensor -> logits (B, 16)."""
        x = x.contiguous()
        B = x.shape[0]
        _lib.check(_lib.lib().fdr_propose_forward(self._h, ptr(x), B, ptr(self._logits),
                                                  stream_handle()))
        return self._logits[:B].clone()

    def probabilities(self, x):
        out = []
        for s in range(0, x.shape[0], self.max_batch):
            out.append(torch.sigmoid(self.forward(x[s:s + self.max_batch])))
        return torch.cat(out)

    def gradients(self, x, labels):
        """(gradient of the mean BCE wrt every parameter, loss) without an update."""
        x, labels = x.contiguous(), labels.contiguous()
        g = torch.empty(self.nparams, dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().fdr_propose_gradients(self._h, ptr(x), ptr(labels), x.shape[0],
                                                    ptr(self._logits), ptr(g), ptr(self._loss),
                                                    stream_handle()))
        return g, float(self._loss.item())

    def train_step(self, x, labels, lr):
        """One Adam step; returns the device loss scalar (no host sync)."""
        x, labels = x.contiguous(), labels.contiguous()
        _lib.check(_lib.lib().fdr_propose_train_step(self._h, ptr(x), ptr(labels), x.shape[0],
                                                     float(lr), ptr(self._logits), ptr(self._loss),
                                                     stream_handle()))
        return self._loss

    # ---- checkpoint / resume ----------------------------------------------------------
    def get_state(self):
        n = self.nparams
        p, m, v = (np.empty(n, np.float32) for _ in range(3))
        step = C.c_int64()
        _lib.check(_lib.lib().fdr_propose_get_state(self._h, p.ctypes.data_as(C.c_void_p),
                                                    m.ctypes.data_as(C.c_void_p),
                                                    v.ctypes.data_as(C.c_void_p), C.byref(step)))
        return {"params": p, "m": m, "v": v, "step": step.value}

    def set_state(self, st):
        p = np.ascontiguousarray(st["params"], np.float32)
        if p.size != self.nparams:
            raise ValueError(f"state has {p.size} parameters, the network {self.nparams}")
        m = np.ascontiguousarray(st["m"] if st.get("m") is not None else np.zeros_like(p), np.float32)
        v = np.ascontiguousarray(st["v"] if st.get("v") is not None else np.zeros_like(p), np.float32)
        _lib.check(_lib.lib().fdr_propose_set_state(self._h, p.ctypes.data_as(C.c_void_p),
                                                    m.ctypes.data_as(C.c_void_p),
                                                    v.ctypes.data_as(C.c_void_p), int(st.get("step", 0))))

    def save(self, path, extra=None):
        """Flat binary: u64 header length, JSON header, then params, m, v (float32 LE)."""
        st = self.get_state()
        hdr = {"format": "fdr_propose_net/1", "nbins": self.nbins, "cin": self.cin, "width": 32,
               "ksize": 5, "nwin": NWIN, "nparams": self.nparams, "step": st["step"],
               "seed": self.seed, "lag": self.lag, "compress": self.compress,
               "extra": dict(self.meta, **(extra or {}))}
        hb = json.dumps(hdr, sort_keys=True).encode()
        with open(path, "wb") as fh:
            fh.write(struct.pack("<Q", len(hb)))
            fh.write(hb)
            for k in ("params", "m", "v"):
                fh.write(st[k].astype("<f4").tobytes())

    @staticmethod
    def read_checkpoint(path):
        with open(path, "rb") as fh:
            n = struct.unpack("<Q", fh.read(8))[0]
            hdr = json.loads(fh.read(n))
            if hdr.get("format") != "fdr_propose_net/1":
                raise ValueError(f"{path}: not a proposal-net checkpoint")
            arrs = [np.frombuffer(fh.read(4 * hdr["nparams"]), "<f4").astype(np.float32)
                    for _ in range(3)]
        return hdr, {"params": arrs[0], "m": arrs[1], "v": arrs[2], "step": hdr["step"]}

    @classmethod
    def load(cls, path, max_batch=64):
        hdr, st = cls.read_checkpoint(path)
        net = cls(hdr["nbins"], hdr["cin"], max_batch=max_batch, seed=hdr["seed"],
                  lag=hdr.get("lag", False), compress=hdr.get("compress", False))
        net.set_state(st)
        net.meta = hdr.get("extra", {})
        return net


def features(spec, lag=False, compress=True, factor=FACTOR, out=None, stream=None):
    """Network input (cin, Nf/factor) of a column-major (Nf, Nt) CUDA spectrogram: the
    power rows, then (lag) the 17 lag-product rows, each value v compressed to
    sign(v)*log1p(|v|) when ``compress``."""
    Nf, Nt = spec.shape
    nb = Nf // factor
    cin = input_channels(Nt, lag)
    if out is None:
        out = torch.empty((cin, nb), dtype=torch.float32, device="cuda")
    if tuple(out.shape) != (cin, nb) or not out.is_contiguous():
        raise ValueError(f"features: out must be a contiguous ({cin}, {nb}) tensor")
    sh = stream_handle(stream)
    cflag = 1 if compress else 0
    if lag:
        _lib.check(_lib.lib().fdr_propose_input(ptr(spec), Nf, Nt, factor, MAXLAG, cflag,
                                                ptr(out), sh))
    else:
        _lib.check(_lib.lib().fdr_propose_features(ptr(spec), Nf, Nt, factor, cflag, ptr(out), sh))
    return out


def synth_channel(seed, Nf=1 << 20, Nt=16, max_tones=5, snr=(8.0, 40.0), rmax=8.0):
    """Seeded synthetic coarse channel on the device: exponential(1) background plus
    0..max_tones drifting tones of per-step amplitude uniform in ``snr`` and rate uniform in
    [-rmax, rmax] ch/step (power split linearly between the two neighbouring channels).
    Returns the column-major (Nf, Nt) spectrogram and the tone list (c0, rate, amplitude)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed))
    spec = torch.rand((Nt, Nf), device="cuda", generator=g).clamp_min_(1e-30).log_().neg_()
    ntones = int(rng.integers(0, max_tones + 1))
    tones = []
    if ntones:
        c0 = rng.uniform(0, Nf, ntones)
        r = rng.uniform(-rmax, rmax, ntones)
        a = rng.uniform(snr[0], snr[1], ntones)
        tones = list(zip(c0.tolist(), r.tolist(), a.tolist()))
        t = np.arange(Nt)
        c = c0[:, None] + r[:, None] * t[None, :]
        lo = np.floor(c)
        f = c - lo
        lo = lo.astype(np.int64) % Nf
        hi = (lo + 1) % Nf
        rows = np.broadcast_to(t[None, :], c.shape)
        idx = np.concatenate([(rows * Nf + lo).ravel(), (rows * Nf + hi).ravel()])
        val = np.concatenate([(a[:, None] * (1 - f)).ravel(), (a[:, None] * f).ravel()])
        spec.view(-1).index_add_(0, torch.from_numpy(idx).cuda(),
                                 torch.from_numpy(val.astype(np.float32)).cuda())
    return spec.t(), tones


class FullSearch:
    """Full-rate plain ZDT (256 rates, -8:1/16:8-1/16) + fused proto-hit scan: the labeller,
    the low-confidence fallback and the reference against which recall is measured."""

    def __init__(self, Nf=1 << 20, Nt=16):
        self.ws = ZDTWorkspace(None, R_MIN, DR, NRATES, shape=(Nf, Nt))
        self.dest = fortran_empty(Nf, NRATES)

    def hits(self, spec, snr=10.0):
        return zdtfdr_protohits_(self.dest, self.ws, spec, threshold=snr, snr=True)


def window_hit_counts(hits):
    """Proto-hits per rate window (length 16)."""
    if len(hits) == 0:
        return np.zeros(NWIN, np.int64)
    return np.bincount(np.asarray(hits)[:, 1] // RATES_PER_WIN, minlength=NWIN)[:NWIN]


def make_batch(seeds, full, lag, Nf=1 << 20, Nt=16, out=None, keep_hits=False, compress=True):
    """Features (B, cin, Nf/256), labels (B, 16) and per-window hit counts (B, 16) for the
    seeded channels ``seeds`` (labels: 1 where the full search finds a proto-hit)."""
    B = len(seeds)
    cin = input_channels(Nt, lag)
    X = out if out is not None else torch.empty((B, cin, Nf // FACTOR), dtype=torch.float32,
                                                device="cuda")
    counts = np.zeros((B, NWIN), np.int64)
    all_hits = []
    for i, sd in enumerate(seeds):
        spec, _ = synth_channel(int(sd), Nf, Nt)
        features(spec, lag, compress, out=X[i])
        h = full.hits(spec)
        counts[i] = window_hit_counts(h)
        if keep_hits:
            all_hits.append(h)
    Y = torch.from_numpy((counts > 0).astype(np.float32)).cuda()
    return (X, Y, counts, all_hits) if keep_hits else (X, Y, counts)


def lr_at(step, total, lr):
    """Cosine decay from lr to lr/20."""
    return lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * min(step, total) / max(1, total))))


def train_online(nets, nchannels, seed0, batch=64, lr=2e-3, full=None, Nf=1 << 20, Nt=16,
                 log=None, log_every=50, start_step=0):
    """Train one or more networks on ``nchannels`` fresh seeded channels (seed0, seed0+1, ...),
    one pass, ``batch`` channels per Adam step; the labels (one full search per channel) are
    shared, a network without ``lag`` reads the power rows only.  Resumable: ``start_step``
    skips the batches already seen.  Returns the loss history [(step, loss per network)]."""
    nets = list(nets) if isinstance(nets, (list, tuple)) else [nets]
    full = full or FullSearch(Nf, Nt)
    total = nchannels // batch
    compress = nets[0].compress
    if any(n.compress != compress for n in nets):
        raise ValueError("networks trained together share the feature compression")
    X = torch.empty((batch, input_channels(Nt, True), Nf // FACTOR), dtype=torch.float32,
                    device="cuda")
    Xp = torch.empty((batch, Nt, Nf // FACTOR), dtype=torch.float32, device="cuda")
    hist = []
    t0 = time.time()
    for step in range(start_step, total):
        seeds = range(seed0 + step * batch, seed0 + (step + 1) * batch)
        _, Y, _ = make_batch(seeds, full, True, Nf, Nt, out=X, compress=compress)
        losses = []
        for n in nets:
            if n.lag:
                losses.append(n.train_step(X, Y, lr_at(step, total, lr)))
            else:
                Xp.copy_(X[:, :Nt])
                losses.append(n.train_step(Xp, Y, lr_at(step, total, lr)))
        if log_every and (step % log_every == 0 or step == total - 1):
            lv = [round(float(l.item()), 5) for l in losses]
            hist.append((step, lv))
            if log:
                log(f"step {step}/{total} loss {lv} ({time.time() - t0:.0f} s)")
    torch.cuda.synchronize()
    return hist


class ProposalSearch:
    """zdtfdr! + findprotohits restricted to the windows the network proposes.

    Per channel, with p_w the window probabilities: windows with p_w >= tau_hi are run; a
    window with tau <= p_w < tau_hi is uncertain, and a channel with any uncertain window
    (or with more than ``max_windows`` windows to run) falls back to the full 256-rate
    search.  The proposed windows run in one pass of the fused kernels over their 8-rate
    blocks (zdtfdr_blocks_protohits_, sharing the full search's workspace); the proto-hit
    threshold is denormalised from the statistics of the columns that ran (findprotohits
    over an iterable of FDR matrices, fdrutils.jl:156-169)."""

    def __init__(self, net, tau=0.05, tau_hi=None, max_windows=NWIN, Nf=1 << 20, Nt=16,
                 full=None):
        self.net = net
        self.tau = tau
        self.tau_hi = tau if tau_hi is None else tau_hi
        self.max_windows = max_windows
        self.Nf, self.Nt = Nf, Nt
        self.full = full or FullSearch(Nf, Nt)

    def decide(self, p):
        """(windows to run, fallback?) for probabilities p (16,)."""
        p = np.asarray(p)
        if np.any((p >= self.tau) & (p < self.tau_hi)):
            return None, True
        wins = np.nonzero(p >= self.tau_hi)[0]
        if len(wins) > self.max_windows:
            return None, True
        return wins, False

    def probabilities(self, specs):
        X = torch.empty((len(specs), self.net.cin, self.Nf // FACTOR), dtype=torch.float32,
                        device="cuda")
        for i, s in enumerate(specs):
            features(s, self.net.lag, self.net.compress, out=X[i])
        return self.net.probabilities(X).cpu().numpy()

    def search(self, spec, p, snr=10.0):
        """(hits with global rate indices, rates computed, fell back?)."""
        wins, fb = self.decide(p)
        if fb:
            return self.full.hits(spec, snr), NRATES, True
        if len(wins) == 0:
            return np.zeros((0, 2), np.int64), 0, False
        per = RATES_PER_WIN // 8
        blocks = (wins[:, None] * per + np.arange(per)[None, :]).ravel()
        dest = self.full.dest[:, :8 * len(blocks)]
        h = zdtfdr_blocks_protohits_(dest, self.full.ws, spec, blocks, threshold=snr, snr=True)
        if len(h):
            h = h.copy()
            h[:, 1] = blocks[h[:, 1] // 8] * 8 + h[:, 1] % 8
        return h, len(wins) * RATES_PER_WIN, False


def recall(hits, ref):
    """|hits & ref| / |ref| over (i, j) pairs (1.0 when ref is empty)."""
    if len(ref) == 0:
        return 1.0
    a = set(map(tuple, np.asarray(hits).tolist()))
    b = set(map(tuple, np.asarray(ref).tolist()))
    return len(a & b) / len(b)


def calibrate(probs, counts, target=0.997, fixed_cost=0.0, win_cost=1.0, full_cost=None):
    """Pick (tau, tau_hi, max_windows) on a validation set so that the proto-hits inside the
    windows that run (or in channels that fall back) are >= ``target`` of all proto-hits, at
    the least modelled cost: fixed_cost + win_cost per window for a channel whose windows
    run (nothing when no window is proposed), full_cost for a fallback (default: 16 windows).
    A channel falls back when a window is uncertain (tau <= p < tau_hi) or when more than
    max_windows windows would run."""
    probs, counts = np.asarray(probs, np.float64), np.asarray(counts)
    full_cost = fixed_cost + NWIN * win_cost if full_cost is None else full_cost
    total = counts.sum()
    ch_hits = counts.sum(axis=1)
    grid = np.unique(np.concatenate([[0.0, 1.0], np.quantile(probs, np.linspace(0, 1, 201))]))
    best = None
    for tau in grid:
        above = probs >= tau
        for tau_hi in grid[grid >= tau]:
            run = probs >= tau_hi
            unc = np.any(above & ~run, axis=1)
            k = run.sum(axis=1)
            in_run = (counts * run).sum(axis=1)
            for kmax in range(NWIN + 1):
                fb = unc | (k > kmax)
                found = np.where(fb, ch_hits, in_run).sum()
                rec = found / total if total else 1.0
                if rec < target:
                    continue
                cost = np.where(fb, full_cost, np.where(k > 0, fixed_cost + k * win_cost, 0.0)).sum()
                if best is None or cost < best[0]:
                    best = (float(cost), float(tau), float(tau_hi), int(kmax), float(rec),
                            float(fb.mean()))
    return {"cost": best[0], "cost_frac": best[0] / (full_cost * len(probs)), "tau": best[1],
            "tau_hi": best[2], "max_windows": best[3], "window_recall": best[4],
            "fallback_rate": best[5]}


def measure_costs(full, spec, reps=10):
    """Device-synchronised wall time (ms) of the full search and of window searches with 1
    and 16 windows on one channel -> (fixed, per-window, full) of the calibration cost model."""
    srch = ProposalSearch(None, tau=0.5, full=full)

    def tm(f):
        f()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(reps):
            f()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) / reps * 1e3

    t_full = tm(lambda: full.hits(spec))
    p1, p16 = np.zeros(NWIN), np.ones(NWIN)
    p1[0] = 1.0
    t1 = tm(lambda: srch.search(spec, p1))
    t16 = tm(lambda: srch.search(spec, p16))
    per = (t16 - t1) / (NWIN - 1)
    return {"fixed_ms": t1 - per, "per_window_ms": per, "full_ms": t_full}


def evaluate(net, specs, full, tau, tau_hi, snr=10.0, ref_hits=None, max_windows=NWIN):
    """Proposal search over ``specs`` (resident CUDA spectrograms) against the full search:
    proto-hit recall (pooled over channels), rates computed, fallbacks and the device-
    synchronised wall time of both paths (the proposal path includes its features and
    network inference; net=None proposes every window)."""
    srch = ProposalSearch(net, tau=tau, tau_hi=tau_hi, max_windows=max_windows, full=full)
    if ref_hits is None:
        ref_hits = [full.hits(s, snr) for s in specs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in specs:
        full.hits(s, snr)
    torch.cuda.synchronize()
    t_full = time.perf_counter() - t0
    t0 = time.perf_counter()
    if net is not None:
        probs = srch.probabilities(specs)
    else:
        probs = np.ones((len(specs), NWIN))
    out = [srch.search(s, p, snr) for s, p in zip(specs, probs)]
    torch.cuda.synchronize()
    t_prop = time.perf_counter() - t0
    found = total = rates = fb = 0
    for (h, nr, f), ref in zip(out, ref_hits):
        total += len(ref)
        if len(ref):
            found += int(round(recall(h, ref) * len(ref)))
        rates += nr
        fb += int(f)
    n = len(specs)
    return {"channels": n, "recall": found / total if total else 1.0, "hits": total,
            "rates_frac": rates / (n * NRATES), "fallback_frac": fb / n,
            "full_ms_per_channel": t_full / n * 1e3, "proposal_ms_per_channel": t_prop / n * 1e3,
            "speedup": t_full / t_prop}
