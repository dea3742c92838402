"""Benchmark of the adaptive MWDG2/HWFV1 time step on B200.

Workload: fBm catchment, 4096 x 4096 finest cells (max_ref_lvl 12),
2 m cells, Hurst 0.8, relief 0-30 m, Manning 0.03, dry start, west-edge point inflow with
a triangular hydrograph peaking at 50 m^3/s at 30 min, epsilon 1e-3, MWDG2, FP32 state
(--precision 64 for FP64). Seeded synthetic DEM (the reference ships no such DEM).

A step is one adaptive time step (MRA encode/threshold/regularise/decode, leaf topology,
both RK stages, CFL dt). Metric: active-cell updates per second = leaves updated per
step, summed over the timed steps, divided by their device time (CUDA events on the
library's stream). Every input and the state are resident in HBM (the hierarchy alone is
~1 GB in FP32, far larger than the 126 MB L2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference algorithm's CPU restatement (the reference itself
has no CPU path; its CUDA build is timed separately) on all host cores.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-mwdg2_b200"))

METRIC = "active-cell updates/s (adaptive MWDG2 time step)"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--solver", default="mwdg2", choices=["mwdg2", "hwfv1"])
    ap.add_argument("--level", type=int, default=12)
    ap.add_argument("--cpu-steps", type=int, default=2, help="timed oracle steps for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case-dir", default=None)
    return ap.parse_args()


def workload(a) -> dict:
    return {"workload": f"fBm catchment {1 << a.level}^2 finest cells (max_ref_lvl {a.level}), 2 m cells, "
                        "Hurst 0.8, relief 0-30 m, Manning 0.03, dry start, west point inflow 50 m3/s peak at 30 min, "
                        "epsilon 1e-3",
            "solver": a.solver, "precision": f"fp{a.precision}", "max_ref_lvl": a.level,
            "steps_from": "simulation start (steps W+1..W+K of the run)",
            "l2": "inputs larger than L2 (hierarchy arrays >= 1 GB)"}


def make_case(a, rank: int) -> str:
    import cases
    key = hashlib.sha1(f"{a.level}-{a.solver}-v1".encode()).hexdigest()[:10]
    base = a.case_dir or os.path.join(tempfile.gettempdir(), "mwdg2_bench_cases")
    d = os.path.join(base, f"{key}-r{rank}")
    par = os.path.join(d, "case.par")
    if os.path.exists(os.path.join(d, "READY")):
        return par
    os.makedirs(d, exist_ok=True)
    cases.fbm_catchment(d, L=a.level, solver=a.solver, eps=1e-3, sim_time=7200.0, cellsize=2.0, hurst=0.8,
                        relief=30.0, manning=0.03, peak_q=50.0, t_peak=1800.0, seed=20261203)
    open(os.path.join(d, "READY"), "w").write("ok\n")
    return par


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self) -> dict:
        rows = []
        try:
            for ln in open(self.path):
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(par: str, a, steps: int) -> dict:
    """The oracle (CPU restatement of the reference algorithm) on this machine's host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    o = oracle_py.Oracle(par, a.precision)
    o.step()  # first step (full encode from the initial grid) is not timed
    n_tot = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        ok, dt, n = o.step()
        n_tot += n
    wall = time.perf_counter() - t0
    o.close()
    return {"value": n_tot / wall, "unit": UNIT, "cores": oracle_py.num_threads(), "kind": "port",
            "sample": f"steps 2..{steps + 1} of the same case ({steps} full adaptive steps, {n_tot} leaf updates, "
                      f"{wall:.1f} s)"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    par = make_case(a, 0)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    o = oracle_py.Oracle(par, a.precision)
    for _ in range(a.warmup):
        o.step()
    n_tot = 0
    t0 = time.perf_counter()
    for _ in range(a.steps):
        ok, dt, n = o.step()
        n_tot += n
    wall = time.perf_counter() - t0
    v = n_tot / wall
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * wall / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"f{a.precision}", "data": "synthetic (seeded fBm DEM)", "config": workload(a),
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": oracle_py.num_threads(), "kind": "port",
                             "sample": f"{a.steps} full adaptive steps after {a.warmup} warm-up steps"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    import numpy as np
    import torch
    import mwdg2_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    par = make_case(a, rank)
    sim = mwdg2_b200.Simulation(par, precision=a.precision, device=local, timing=True)
    clk = Clocks(local).__enter__()   # sampled from the warm-up through the end-to-end loop
    for _ in range(a.warmup):
        sim.step()

    # device-timed steps (replicas: every rank runs the same workload on its own GPU)
    barrier()
    ms_step, ms_phase, leaves, counters = [], [], [], []
    for _ in range(a.steps):
        ok, dt, n = sim.step()
        t = sim.last_step_timing()
        ms_step.append(float(t[7]))
        ms_phase.append(t.tolist())
        leaves.append(n)
        counters.append(sim.last_step_counters())
    barrier()
    tot_ms = float(sum(ms_step))
    if dist:
        tt = torch.tensor([tot_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms = float(tt.item())
    value = world * sum(leaves) / (tot_ms / 1e3)

    # end to end through the C ABI: each step's inputs (point-source values) go host->device
    # from pinned memory inside mwdg2_step, its scalars come back, and the stage-point
    # depths are read into a host buffer (mwdg2_read_stage)
    n_pts = 2
    barrier()
    t0 = time.perf_counter()
    e2e_leaves = 0
    for _ in range(a.steps):
        ok, dt, n = sim.step()
        sim.stage(n_pts)
        e2e_leaves += n
    barrier()
    e2e_wall = time.perf_counter() - t0
    clk.__exit__(None, None, None)
    if dist:
        tt = torch.tensor([e2e_wall], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_wall = float(tt.item())
    P = a.precision // 8
    h2d = 1 * (8 + P)            # one point source record {code, type, value}
    d2h = (6 * P + 8 + 24) + 4 * P * n_pts

    # roofline of the dominant kernel, from its live event timing
    ph = np.array(ms_phase)
    mean_ph = ph.mean(axis=0)
    n_mean = float(np.mean(leaves))
    peak, peak_kind = peaks()
    # per-leaf compulsory bytes of a fused MWDG2 stage kernel: topology 25 B (act, level,
    # 4 neighbour ids + levels) + own 12 coefficients read + 18 written (stage 1: U^n, U*;
    # stage 2: U^n read and written) = 25 + 30P
    cand = {"k_mwdg2_stage<1> (RK stage 1: gather, friction, limiter, DG2)": (mean_ph[4], 25 + 30 * P),
            "k_mwdg2_stage<2> (RK stage 2: gather, limiter, DG2, RK average, CFL)": (mean_ph[6], 25 + 30 * P)}
    if a.solver == "hwfv1":
        cand = {"k_hwfv1 (gather, friction, FV1 update, CFL)": (mean_ph[4], 25 + 7 * P)}
    kname, (kms, per_leaf) = max(cand.items(), key=lambda kv: kv[1][0])
    achieved = per_leaf * n_mean / (kms / 1e3) / 1e9
    c = counters[-1]
    step_bytes = (c["encoded"] * (73 * P + 1) + c["reencoded"] * 45 * P + c["detail_slots"] * (P + 2) +
                  c["decoded"] * 72 * P + 40 * n_mean + n_mean * (51 * P + 32))
    step_gbs = step_bytes / (statistics.mean(ms_step) / 1e3) / 1e9

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": tot_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"f{a.precision}", "data": "synthetic (seeded fBm DEM, no network)", "config": workload(a),
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                         "bytes_per_leaf": per_leaf, "leaves_per_launch": n_mean, "kernel_ms": kms},
            "roofline_step": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_gbs, "frac": step_gbs / peak},
            "e2e": {"value": world * e2e_leaves / e2e_wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(sum(cc["launches"] for cc in counters)),
            "clocks": clk.summary(),
            "phase_ms_mean": dict(zip(("step_begin_srcs", "encode", "decode", "topology", "stage1",
                                       "reencode", "stage2", "step"), [round(x, 4) for x in mean_ph])),
            "leaves_mean": n_mean}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(par, a, a.cpu_steps)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
