"""Train, calibrate and evaluate the drift-rate window proposal networks.

    python frequencydriftratetransforms.jl_b200/train_proposal.py --channels 200000 \
        --out-dir frequencydriftratetransforms.jl_b200/data

Trains two networks on the same online stream of seeded synthetic channels (Nf=2^20, Nt=16,
0-5 tones of per-step amplitude 8-40 drifting -8..8 ch/step; labels from the full 256-rate
ZDT + findprotohits at SNR 10): ``proposal_lag.bin`` (power + lag-product input) and
``proposal_power.bin`` (power input only).  Their thresholds are calibrated on held-out
channels for a proto-hit recall target under the measured cost of each search; the held-out
test set (256 channels) then reports recall, rates computed and the speed-up over the full
search, next to the untrained network.  Checkpoints carry the thresholds and the report.
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import __graft_entry__  # noqa: E402  (loads the package from this directory)

fdr = __graft_entry__.load_package()
P = fdr.proposal

import numpy as np  # noqa: E402
import torch  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--channels", type=int, default=200_000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--val", type=int, default=512)
    ap.add_argument("--test", type=int, default=256)
    ap.add_argument("--target", type=float, default=0.998, help="calibration recall target")
    ap.add_argument("--out-dir", default=os.path.join(HERE, "data"))
    ap.add_argument("--report", default=None)
    ap.add_argument("--eval-only", default=None, metavar="DIR",
                    help="skip training: load proposal_lag.bin / proposal_power.bin from DIR")
    a = ap.parse_args(argv)
    os.makedirs(a.out_dir, exist_ok=True)
    full = P.FullSearch()
    cin_lag = P.input_channels(16, True)
    nets = {"lag": P.ProposalNet(4096, cin_lag, max_batch=max(a.batch, 64), seed=a.seed, lag=True),
            "power": P.ProposalNet(4096, 16, max_batch=max(a.batch, 64), seed=a.seed, lag=False)}
    untrained = {"lag": P.ProposalNet(4096, cin_lag, max_batch=64, seed=a.seed, lag=True)}
    t0 = time.time()
    if a.eval_only:
        nets = {k: P.ProposalNet.load(os.path.join(a.eval_only, f"proposal_{k}.bin"), max_batch=64)
                for k in ("lag", "power")}
        hist = []
        a.channels = nets["lag"].meta.get("train_channels", a.channels)
    else:
        hist = P.train_online([nets["lag"], nets["power"]], a.channels, 1_000_000, batch=a.batch,
                              lr=a.lr, full=full, log=lambda m: print(m, flush=True), log_every=200)
    train_s = time.time() - t0
    # calibration set
    vseeds = range(2_000_000_000, 2_000_000_000 + a.val)
    Xv, _, cv = P.make_batch(vseeds, full, True)
    spec0, _ = P.synth_channel(int(vseeds[0]))
    costs = P.measure_costs(full, spec0)
    print("costs", costs, flush=True)
    # test set (resident)
    tseeds = range(3_000_000_000, 3_000_000_000 + a.test)
    specs = [P.synth_channel(int(s))[0] for s in tseeds]
    ref = [full.hits(s) for s in specs]
    report = {"train_channels": a.channels, "train_s": train_s, "loss_tail": hist[-5:],
              "costs": costs, "target": a.target, "test_channels": a.test}
    report["no_network"] = P.evaluate(None, specs, full, 0.0, 0.0, ref_hits=ref)
    for name, net in list(nets.items()) + [("untrained_lag", untrained["lag"])]:
        x = Xv if net.lag else Xv[:, :16].contiguous()
        probs = net.probabilities(x).cpu().numpy()
        cal = P.calibrate(probs, cv, target=a.target, fixed_cost=costs["fixed_ms"],
                          win_cost=costs["per_window_ms"], full_cost=costs["full_ms"])
        res = P.evaluate(net, specs, full, cal["tau"], cal["tau_hi"], ref_hits=ref,
                         max_windows=cal["max_windows"])
        report[name] = {"calibration": cal, "test": res}
        print(name, json.dumps(report[name]), flush=True)
        if name in nets:
            net.meta = {"tau": cal["tau"], "tau_hi": cal["tau_hi"],
                        "max_windows": cal["max_windows"], "calibration": cal,
                        "test": res, "train_channels": a.channels, "costs": costs}
            net.save(os.path.join(a.out_dir, f"proposal_{name}.bin"))
    print(json.dumps(report), flush=True)
    if a.report:
        with open(a.report, "w") as fh:
            json.dump(report, fh, indent=1)


if __name__ == "__main__":
    main()
