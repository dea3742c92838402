"""Train the learned refinement proposal's MLP on plain MWDG2 runs.

Each training scenario is a seeded 1024 x 1024 fBm catchment (max_ref_lvl 10, 2 m cells,
Hurst U(0.6, 0.9), relief 0-30 m, Manning U(0.02, 0.04), epsilon 1e-3) driven, with equal
chance, by a west-edge point inflow peaking at U(20, 50) m^3/s or by a dam break of random
radius over part of the domain. The plain step runs on the GPU with the proposal's
recording on (mwdg2_proposal_record): at the start of every step the features of every
coarse cell (8 x 8 finest cells) are built on the device, and at its end each child
subtree's activity (a leaf the RK stages updated, or its significance flags changed since
the last step). Every `--every`-th step one Adam step of the tcgen05 training kernel is taken on
all coarse cells of that step (mwdg2_trainer_observe), with the active class weighted by
`--pos-weight`. The last `--holdout` scenarios are not trained on: every step of them scores
the trained proposal (at the chosen logit threshold) against the step's activity on the
device, and the parameters are written with its recall and precision to proposal_mlp.npz.

    python gpu-mwdg2_b200/train_proposal.py [--scenarios 200] [--sim-time 900] ...
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases  # noqa: E402
import mwdg2_b200  # noqa: E402


def scenario(root: str, i: int, seed: int, L: int, sim_time: float) -> str:
    rng = np.random.Generator(np.random.PCG64(seed + 7919 * i))
    hurst = float(rng.uniform(0.6, 0.9))
    manning = float(rng.uniform(0.02, 0.04))
    d = os.path.join(root, f"s{i:03d}")
    n = 1 << L
    if rng.random() < 0.5:
        c = cases.fbm_catchment(d, L=L, sim_time=sim_time, hurst=hurst, manning=manning,
                                peak_q=float(rng.uniform(20.0, 50.0)), t_peak=float(rng.uniform(200.0, 600.0)),
                                seed=seed + i)
    else:
        z = cases.fbm_surface(n, hurst, seed + i, 30.0)
        cx, cy = rng.uniform(0.2, 0.8, size=2) * n
        r = float(rng.uniform(0.05, 0.2)) * n
        Y, X = np.mgrid[0:n, 0:n]
        level = float(np.percentile(z, rng.uniform(30.0, 70.0)))
        h0 = np.where(np.hypot(X - cx, Y - cy) < r, np.maximum(0.0, level + 3.0 - z), 0.0)
        c = cases.fbm_catchment(d, L=L, sim_time=sim_time, hurst=hurst, manning=manning, peak_q=0.0, t_peak=300.0,
                                seed=seed + i, start_depth=h0)
    return c.par


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenarios", type=int, default=200)
    ap.add_argument("--holdout", type=int, default=10)
    ap.add_argument("--level", type=int, default=10)
    ap.add_argument("--sim-time", type=float, default=900.0)
    ap.add_argument("--every", type=int, default=10, help="steps between Adam steps")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--pos-weight", type=float, default=4.0)
    ap.add_argument("--threshold", type=float, default=-2.0, help="logit threshold of the proposal")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--out", default=os.path.join(HERE, "proposal_mlp.npz"))
    a = ap.parse_args()
    t0 = time.time()
    tr = mwdg2_b200.Trainer(mwdg2_b200.mlp_init(a.seed), lr=a.lr)
    losses, n_steps, n_updates = [], 0, 0
    counts = np.zeros(4)   # true positive, false negative, false positive, true negative (holdout)
    with tempfile.TemporaryDirectory() as root:
        for i in range(a.scenarios):
            par = scenario(root, i, a.seed, a.level, a.sim_time)
            hold = i >= a.scenarios - a.holdout
            sim = mwdg2_b200.Simulation(par, precision=a.precision)
            sim.proposal_record(True)
            if hold:
                # every step a judge step: the proposal is scored against the step's activity
                # on the device and never applied
                sim.proposal_enable(tr.params(), judge_every=1, threshold=a.threshold, miss_bound=1.0)
            k = 0
            while True:
                ok, dt, n = sim.step()
                if not ok:
                    break
                k += 1
                n_steps += 1
                if k < 2:
                    continue
                if hold:
                    st = sim.proposal_stats()
                    tp = st["active"] - st["missed"]
                    counts += [tp, st["missed"], st["proposed"] - tp, st["subtrees"] - st["proposed"] - st["missed"]]
                elif k % a.every == 0:
                    losses.append(tr.observe(sim, a.pos_weight))
                    n_updates += 1
            sim.close()
            shutil.rmtree(os.path.dirname(par), ignore_errors=True)
            if (i + 1) % 10 == 0:
                print(json.dumps({"scenarios": i + 1, "steps": n_steps, "updates": n_updates,
                                  "loss_recent": float(np.mean(losses[-100:])) if losses else None,
                                  "seconds": round(time.time() - t0, 1)}), flush=True)
    params = tr.params()
    tr.close()
    tp, fn, fp, tn = counts
    summary = {"scenarios": a.scenarios, "holdout": a.holdout, "level": a.level, "sim_time": a.sim_time,
               "every": a.every, "lr": a.lr, "pos_weight": a.pos_weight, "threshold": a.threshold,
               "precision": a.precision, "steps": n_steps, "updates": n_updates,
               "loss_first": float(np.mean(losses[:50])) if losses else None,
               "loss_last": float(np.mean(losses[-200:])) if losses else None,
               "holdout_recall": float(tp / max(1.0, tp + fn)), "holdout_precision": float(tp / max(1.0, tp + fp)),
               "holdout_proposed_fraction": float((tp + fp) / max(1.0, counts.sum())),
               "holdout_active_fraction": float((tp + fn) / max(1.0, counts.sum())),
               "seconds": round(time.time() - t0, 1)}
    np.savez(a.out, params=params, summary=json.dumps(summary))
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
