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
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (catchment: 1000, a window of about 0.6 s on the device; others: 20)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--solver", default="mwdg2", choices=["mwdg2", "hwfv1"])
    ap.add_argument("--level", type=int, default=None, help="max_ref_lvl (catchment 12, urban 13)")
    ap.add_argument("--cpu-steps", type=int, default=16, help="timed FP64 oracle steps for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case-dir", default=None)
    ap.add_argument("--workload", default="catchment", choices=["catchment", "urban", "ensemble", "learned"],
                    help="urban: 8192^2 fBm base with building blocks, lake at rest at 1 m, rising point "
                         "inflow; ensemble: a batch of seeded uneven scenarios (mwdg2_batch_*) against the "
                         "same members stepped one after another; learned: the catchment run to --eval-time "
                         "plain in FP64 and FP32 and with the learned refinement proposal in FP32; each of "
                         "the last two prints its own line")
    ap.add_argument("--eval-time", type=float, default=1800.0, help="learned: simulated seconds of the runs")
    ap.add_argument("--judge-every", type=int, default=20, help="learned: steps between judge steps")
    ap.add_argument("--proposal", default=os.path.join(ROOT, "gpu-mwdg2_b200", "proposal_mlp.npz"),
                    help="learned: trained MLP parameters")
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--decode", default="reference", choices=["reference", "keep"],
                    help="decode of the timed run (mwdg2_set_decode_mode): reference (bit for bit the "
                         "reference build's) or keep (children of encoded parents keep their values); the "
                         "catchment line also carries a keep-values window beside the reference one")
    ap.add_argument("--peak-time", type=float, default=1800.0,
                    help="catchment: a second timing window starting at this simulated time (the hydrograph "
                         "peak); <= 0 skips it")
    a = ap.parse_args()
    if a.level is None:
        a.level = 13 if a.workload == "urban" else 12
    if a.steps is None:
        a.steps = 1000 if a.workload == "catchment" else 20
    return a


def workload(a) -> dict:
    if a.workload == "urban":
        return {"workload": f"urban catchment {1 << a.level}^2 finest cells (max_ref_lvl {a.level}), 1 m cells, "
                            "fBm base Hurst 0.8 relief 0-3 m plus axis-aligned blocks 8-30 cells wide and "
                            "5-20 m tall on ~30 % of the area, lake at rest at 1 m, Manning 0.03, west point "
                            "inflow rising 0-100 m3/s over 15 min, epsilon 1e-3",
                "solver": a.solver, "precision": f"fp{a.precision}", "max_ref_lvl": a.level,
                "steps_from": "simulation start (steps W+1..W+K of the run)",
                "l2": "inputs larger than L2 (hierarchy arrays >= 4 GB)"}
    return {"workload": f"fBm catchment {1 << a.level}^2 finest cells (max_ref_lvl {a.level}), 2 m cells, "
                        "Hurst 0.8, relief 0-30 m, Manning 0.03, dry start, west point inflow 50 m3/s peak at 30 min, "
                        "epsilon 1e-3",
            "solver": a.solver, "precision": f"fp{a.precision}", "max_ref_lvl": a.level,
            "decode": getattr(a, "decode", "reference"),
            "steps_from": "simulation start (steps W+1..W+K of the run)",
            "l2": "inputs larger than L2 (hierarchy arrays >= 1 GB)"}


def make_case(a, rank: int) -> str:
    import cases
    key = hashlib.sha1(f"{a.workload}-{a.level}-{a.solver}-v1".encode()).hexdigest()[:10]
    base = a.case_dir or os.path.join(tempfile.gettempdir(), "mwdg2_bench_cases")
    d = os.path.join(base, f"{key}-r{rank}")
    par = os.path.join(d, "case.par")
    if os.path.exists(os.path.join(d, "READY")):
        return par
    os.makedirs(d, exist_ok=True)
    if a.workload == "urban":
        cases.urban_catchment(d, L=a.level, solver=a.solver, eps=1e-3, sim_time=3600.0, cellsize=1.0,
                              lake_level=1.0, peak_q=100.0, t_rise=900.0, manning=0.03, seed=20261203)
    else:
        cases.fbm_catchment(d, L=a.level, solver=a.solver, eps=1e-3, sim_time=7200.0, cellsize=2.0, hurst=0.8,
                            relief=30.0, manning=0.03, peak_q=50.0, t_peak=1800.0, seed=20261203)
    open(os.path.join(d, "READY"), "w").write("ok\n")
    return par


class Clocks:
    """SM clock and clock-event reasons sampled through NVML (read-only queries) on a
    background thread every ~2 ms from the warm-up to the end of the end-to-end loop."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device: int):
        self.device = device
        self.rows: list[tuple[float, float, int]] = []
        self._stop = None
        self._thread = None

    def _handle(self, nv):
        """NVML handle of this process's CUDA device (CUDA and NVML orderings can differ)."""
        import torch
        p = torch.cuda.get_device_properties(self.device)
        try:
            return nv.nvmlDeviceGetHandleByUUID(f"GPU-{p.uuid}".encode())
        except Exception:
            pass
        try:
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception:
            return self
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                    self.rows.append((sm, mx, rs))
                except Exception:
                    pass
                self._stop.wait(0.002)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        reasons = sorted({n for _, _, r in self.rows for n, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": reasons, "samples": len(self.rows), "source": "nvml"}


# DRAM bytes per leaf (dram__bytes_read.sum + dram__bytes_write.sum of the phase's kernels,
# summed, divided by the step's leaves) from a one-pass ncu launch list of this workload
# (4096^2, FP32, 3.0 M leaves). Keyed by (solver, P, timing phase).
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the phase's kernels (one kernel, three "
                  "launches per capture) on the 2048^2 catchment (max_ref_lvl 11, 1.21 M leaves), per leaf, "
                  "x this run's leaves")
PHASE_STEPS = 5
REF_CPU_STEPS = 20   # the reference arm's timed steps on the host cores (at most)
# DRAM bytes per leaf of the RK stages (phase 4: stage 1, phase 6: stage 2) in FP32
TRAFFIC_B_PER_LEAF: dict = {("mwdg2", 4, 4): 181.0, ("mwdg2", 4, 6): 141.6}


def max_over_ranks(x: float, dist, device: str) -> float:
    """The largest per-rank value of x (the slowest replica's time) on every rank; x itself
    without a process group. Every rank must call it at the same point."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, leaves_per_rank: int, max_ms: float) -> float:
    """Whole-job active-cell updates/s of `world` replicas of the same workload: every rank
    updates `leaves_per_rank` leaves over the timed steps, and the job takes as long as the
    slowest rank (`max_ms`, milliseconds)."""
    return world * leaves_per_rank / (max_ms / 1e3)


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_timing(par: str, steps: int, warmup: int) -> dict:
    """The oracle (the reference algorithm restated in C++ with OpenMP) in FP64 -- the
    plain stepper the CPU baseline is defined on -- on this machine's host cores: `warmup`
    untimed steps (the first is the full encode from the initial grid), then `steps` timed
    ones: active-cell updates/s and wall seconds per simulated second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    o = oracle_py.Oracle(par, 64)
    try:
        for _ in range(max(1, warmup)):
            o.step()
        t_sim0 = o.info()["current_time"]
        n_tot = 0
        t0 = time.perf_counter()
        for _ in range(steps):
            ok, dt, n = o.step()
            n_tot += n
        wall = time.perf_counter() - t0
        t_sim = o.info()["current_time"] - t_sim0
    finally:
        o.close()
    return {"value": n_tot / wall, "unit": UNIT, "cores": oracle_py.num_threads(), "kind": "port",
            "dtype": "f64", "cpu_model": cpu_model(), "wall_s": wall, "leaf_updates": n_tot,
            "wall_s_per_sim_s": wall / t_sim if t_sim > 0 else None,
            "sample": f"steps {max(1, warmup) + 1}..{max(1, warmup) + steps} of the same case in FP64 "
                      f"({steps} full adaptive steps, {n_tot} leaf updates, {wall:.1f} s on "
                      f"{oracle_py.num_threads()} OpenMP threads)"}


def cpu_baseline(par: str, a, steps: int) -> dict:
    """The FP64 oracle on the host cores, for the line of this build's own arm."""
    return oracle_timing(par, steps, 1)


def run_reference(a):
    """The reference arm: the reference algorithm on the host cores (it has no CPU path of
    its own, so its FP64 restatement, the oracle port, stands in), timed on this arm's
    workload; beside it, the reference's own CUDA build (oracle/_ref, its unmodified sources
    compiled for sm_100a) on the same case, steps and warm-up in the arm's precision."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    par = make_case(a, 0)
    # a bounded sample of the workload on the host cores (about half a second per step)
    cpu_steps = min(a.steps, REF_CPU_STEPS)
    cpu = oracle_timing(par, cpu_steps, a.warmup)
    v = cpu["value"]
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * cpu["wall_s"] / cpu_steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded fBm DEM)", "config": workload(a),
            "impl": "reference",
            "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model", "dtype")},
            "wall_s_per_sim_s": cpu["wall_s_per_sim_s"],
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import time_reference_build
    try:
        line["reference_cuda"] = time_reference_build.time_reference(par, a.precision, a.steps, a.warmup)
    except Exception as e:   # the binary is missing or the run failed: say so, keep the CPU line
        line["reference_cuda"] = {"unavailable": f"{type(e).__name__}: {str(e)[:300]}"}
    if a.workload == "catchment" and a.peak_time > 0:
        try:
            line["reference_cuda_peak"] = time_reference_build.time_reference(par, a.precision, a.steps, a.warmup,
                                                                              window_time=a.peak_time)
        except Exception as e:
            line["reference_cuda_peak"] = {"unavailable": f"{type(e).__name__}: {str(e)[:300]}"}
    print(json.dumps(line), flush=True)


def run_ensemble(a):
    """Batched ensemble: `--members` seeded scenarios (512^2 to 2048^2 fBm catchments, dam
    breaks or point inflows, Manning n and epsilon drawn per member) advanced together by
    mwdg2_batch_step, against the same members each stepped alone, one after another. Both
    are timed on the host clock around synchronised loops (the batch has one stream per
    member); a step of a member updates its leaves once. Every member takes W warm-up steps,
    then K timed steps (members that reach their end time stop earlier). With --decode keep
    both take the keep-values decode, and the line adds the same members stepped one after
    another with the reference decode (the plain form)."""
    import numpy as np
    import torch
    import cases
    import mwdg2_b200
    torch.cuda.set_device(0)
    base = a.case_dir or os.path.join(tempfile.gettempdir(), "mwdg2_bench_cases")
    root = os.path.join(base, f"ensemble-{a.members}-{a.solver}-v1")
    if not os.path.exists(os.path.join(root, "READY")):
        os.makedirs(root, exist_ok=True)
        cases.ensemble(root, n=a.members, solver=a.solver)
        open(os.path.join(root, "READY"), "w").close()
    pars = sorted(os.path.join(root, d, "case.par") for d in os.listdir(root) if d.startswith("member"))
    sizes = [1 << (int(open(p).read().split("max_ref_lvl")[1].split()[0])) for p in pars]

    with mwdg2_b200.Batch(pars, precision=a.precision) as b:
        for i in range(len(pars)):
            b.member(i).set_decode_mode(a.decode)
        for _ in range(a.warmup):
            b.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        upd, member_steps = 0, 0
        for _ in range(a.steps):
            k, _, n = b.step()
            upd += int(n.sum())
            member_steps += k
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0

    def sequential(mode):
        t_seq, upd_seq = 0.0, 0
        for p in pars:
            s = mwdg2_b200.Simulation(p, precision=a.precision)
            s.set_decode_mode(mode)
            for _ in range(a.warmup):
                s.step()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(a.steps):
                ok, _, n = s.step()
                if not ok:
                    break
                upd_seq += n
            torch.cuda.synchronize()
            t_seq += time.perf_counter() - t0
            s.close()
        return t_seq, upd_seq

    t_seq, upd_seq = sequential(a.decode)
    line = {"metric": "active-cell updates/s (batched ensemble of adaptive MWDG2 time steps)",
            "value": upd / t_batch, "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "impl": "ours-batch", "dtype": f"f{a.precision}",
            "data": "synthetic (seeded fBm DEMs, no network)",
            "config": {"workload": f"ensemble of {a.members} seeded scenarios: finest grids 512^2/1024^2/2048^2 "
                                   "(uniform), fBm Hurst U(0.6,0.9), dam break (radius U(0.05,0.25) x domain, "
                                   "2.5/0.5 m) or point inflow (peak U(5,40) m3/s), n U(0.01,0.05), "
                                   "epsilon {1e-3,1e-4}", "solver": a.solver, "members": len(pars),
                       "grids": {str(m): sizes.count(m) for m in sorted(set(sizes))},
                       "timing": "host clock around synchronised loops"},
            "batch": {"seconds": t_batch, "member_steps": member_steps, "leaf_updates": upd},
            "sequential": {"value": upd_seq / t_seq, "seconds": t_seq, "leaf_updates": upd_seq},
            "batch_over_sequential": (upd / t_batch) / (upd_seq / t_seq), "decode": a.decode}
    if a.decode != "reference":
        t_ref, upd_ref = sequential("reference")
        line["sequential_reference_decode"] = {"value": upd_ref / t_ref, "seconds": t_ref, "leaf_updates": upd_ref}
        line["batch_over_sequential_reference_decode"] = (upd / t_batch) / (upd_ref / t_ref)
    print(json.dumps(line), flush=True)


class nvtx_range:
    """An NVTX range around a timed loop (a no-op without CUDA), so a profiler can capture
    exactly those launches (ncu --nvtx --nvtx-include "<name>/")."""

    def __init__(self, name: str):
        self.name = name
        self.on = False

    def __enter__(self):
        import torch
        self.on = torch.cuda.is_available()
        if self.on:
            torch.cuda.nvtx.range_push(self.name)
        return self

    def __exit__(self, *exc):
        if self.on:
            import torch
            torch.cuda.nvtx.range_pop()


def peak_window(sim, a, dist) -> dict:
    """The same run later on: steps (untimed) until the simulated time reaches a.peak_time,
    then W warm-up steps and K steps timed as the first window (two CUDA events around each
    step): active-cell updates/s, ms per step, wall seconds per simulated second and the
    fraction of leaves that are wet in each RK stage."""
    import numpy as np
    sim.set_timing("step")
    t0 = time.perf_counter()
    advance = 0
    while sim.info()["time"] < a.peak_time:
        ok, dt, n = sim.step()
        if not ok:
            return {"unavailable": f"the run ended before t = {a.peak_time} s"}
        advance += 1
    advance_s = time.perf_counter() - t0
    for _ in range(a.warmup):
        sim.step()
    t_sim0 = sim.info()["time"]
    ms, leaves, wet = [], [], []
    with nvtx_range("peak_window"):
        for _ in range(a.steps):
            ok, dt, n = sim.step()
            ms.append(float(sim.last_step_timing()[7]))
            leaves.append(n)
            c = sim.last_step_counters()
            wet.append((c["wet_stage1"], c["wet_stage2"]))
    sim_s = sim.info()["time"] - t_sim0
    end_time, end_depth = sim.info()["time"], finest_depth(sim)   # for the learned run's comparison
    end_volume = wet_volume(sim)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    tot_ms = max_over_ranks(float(sum(ms)), dist, "cuda")
    n_mean = float(np.mean(leaves))
    # phase breakdown in the window (events between the phases; its first step captures)
    sim.set_timing("phases")
    sim.step()
    ph = []
    for _ in range(PHASE_STEPS):
        sim.step()
        ph.append(sim.last_step_timing().tolist())
    mean_ph = np.array(ph).mean(axis=0)
    return {"from_time": a.peak_time, "steps_to_reach": advance, "seconds_to_reach": advance_s,
            "phase_ms_mean": dict(zip(("step_open", "encode", "decode", "topology", "stage1", "reencode", "stage2",
                                       "step"), [round(float(x), 4) for x in mean_ph])),
            "time_at_window": t_sim0, "value": replica_throughput(world, sum(leaves), tot_ms),
            "ms_per_step": tot_ms / a.steps, "leaves_mean": n_mean,
            "wet_fraction": [float(np.mean([w[k] for w in wet])) / n_mean for k in (0, 1)],
            "wall_s_per_sim_s": (tot_ms / 1e3) / sim_s if sim_s > 0 else None, "sim_seconds": sim_s,
            "timing": "device time of each step (CUDA events on the library's stream), max over ranks",
            "wet_volume_m3": end_volume, "_end_time": end_time, "_end_depth": end_depth}


def wet_volume(sim, tol_h: float = 1e-3) -> float:
    """Water volume (m^3) in the leaves at least tol_h deep: the depths below tol_h in the
    dry area are the multiresolution representation's rounding of eta = h + z over rough
    terrain (a few 1e-6 m per cell in FP32, of either sign, accumulating over a run), which
    would otherwise dominate the total."""
    import numpy as np
    info = sim.info()
    st, lv = sim.state(), sim.leaves()
    area = info["dx"] ** 2 * np.ldexp(1.0, 2 * (info["L"] - lv["lvl"].astype(np.int64)))
    h = st["h0"]
    return float(np.sum(np.where(h >= tol_h, h, 0.0) * area))


def finest_depth(sim):
    """Depth at the centre of every finest cell (Z order) from the leaves' DG2 modes: h0 +
    sqrt(3) (h1x (2 xu - 1) + h1y (2 yu - 1)) at the cell's local coordinates (xu, yu) in
    its leaf (output/write_all_raster_maps_dg2.cu evaluates the same basis)."""
    import numpy as np
    L = sim.info()["L"]
    lv, st = sim.leaves(), sim.state()
    lvl = lv["lvl"].astype(np.int64)
    first = ((1 << (2 * lvl)) - 1) // 3 + 3
    code = lv["act"].astype(np.int64) - first
    span = np.int64(1) << (2 * (L - lvl))
    rep = np.repeat(np.arange(lvl.size), span)
    fz = np.arange(1 << (2 * L), dtype=np.int64)

    def compact(v):
        v = v & 0x55555555
        v = (v | (v >> 1)) & 0x33333333
        v = (v | (v >> 2)) & 0x0F0F0F0F
        v = (v | (v >> 4)) & 0x00FF00FF
        return (v | (v >> 8)) & 0x0000FFFF
    side = (np.int64(1) << (L - lvl))[rep].astype(np.float64)
    x0 = compact(code << (2 * (L - lvl)))[rep]
    y0 = compact((code << (2 * (L - lvl))) >> 1)[rep]
    xu = (compact(fz) - x0 + 0.5) / side
    yu = (compact(fz >> 1) - y0 + 0.5) / side
    s3 = np.sqrt(3.0)
    return st["h0"][rep] + st["h1x"][rep] * s3 * (2 * xu - 1) + st["h1y"][rep] * s3 * (2 * yu - 1)


def par_ending_at(par: str, t_end: float) -> str:
    """A copy of the case's .par (same folder, so its relative paths hold) with sim_time =
    t_end: a run of it takes the same steps as the original and shortens its last step to
    land exactly on t_end (run_simulation.cu:228-235)."""
    out = os.path.join(os.path.dirname(par), "to_%.9g.par" % t_end)
    lines = []
    for line in open(par).read().splitlines():
        w = line.split()
        lines.append(f"sim_time {t_end!r}" if w and w[0] == "sim_time" else line)
    with open(out, "w") as fp:
        fp.write("\n".join(lines) + "\n")
    return out


def learned_window(a, par, t_from, t_end, depth_plain, value_plain, name, volume_plain=None,
                   mode="learned") -> dict:
    """A window of the plain run again with the learned refinement proposal (mode "learned")
    or with the keep-values decode (mode "keep"): a second simulation of the same case
    (ending at t_end, where the plain run's window ended), for "learned" with the trained MLP
    choosing the subtrees the step visits (judge every --judge-every steps), stepped untimed to
    t_from, then W warm-up and K timed steps as the plain window's; its active-cell updates/s,
    and after stepping on to t_end the largest depth difference from the plain run at t_end
    over every finest cell (cell-centre depths). Both take the decode of --decode."""
    import numpy as np
    import mwdg2_b200
    sim = mwdg2_b200.Simulation(par_ending_at(par, t_end), precision=a.precision, timing="step")
    if a.decode == "keep":
        sim.set_decode_mode("keep")
    if mode == "learned":
        z = np.load(a.proposal)
        train = json.loads(str(z["summary"]))
        sim.proposal_enable(z["params"], judge_every=a.judge_every, threshold=train["threshold"], miss_bound=0.02)
    else:
        sim.set_decode_mode("keep")
    ok = True
    while ok and sim.info()["time"] < t_from:
        ok = sim.step()[0]
    for _ in range(a.warmup):
        ok = ok and sim.step()[0]
    ms, leaves, wet = [], [], []
    with nvtx_range(name):
        for _ in range(a.steps):
            ok, dt, n = sim.step()
            if not ok:
                break
            ms.append(float(sim.last_step_timing()[7]))
            leaves.append(n)
            c = sim.last_step_counters()
            wet.append((c["wet_stage1"], c["wet_stage2"]))
    st = sim.proposal_stats() if mode == "learned" else None
    while ok:
        ok = sim.step()[0]
    diff = float(np.max(np.abs(finest_depth(sim) - depth_plain)))
    t_done = sim.info()["time"]
    volume = wet_volume(sim)
    sim.close()
    v = sum(leaves) / (sum(ms) / 1e3)
    n_mean = float(np.mean(leaves))
    out = {"value": v, "ms_per_step": sum(ms) / len(ms), "steps": len(ms), "vs_plain": v / value_plain,
           "leaves_mean": n_mean, "wet_fraction": [float(np.mean([w[k] for w in wet])) / n_mean for k in (0, 1)],
           "max_depth_diff_vs_plain_m": diff, "compared_at_time": t_done, "plain_time": t_end,
           "wet_volume_m3": volume, "plain_wet_volume_m3": volume_plain,
           "timing": "device time of each step (CUDA events) of a second run of the same case, the plain "
                     "window's W warm-up and K timed steps from its start time"}
    if mode == "learned":
        out["proposal"] = {k: st[k] for k in ("active", "proposed", "subtrees", "learned_steps", "judge_steps",
                                               "fallbacks", "frozen_leaves")}
        out["mlp"] = os.path.basename(a.proposal)
        out["judge_every"] = a.judge_every
    else:
        out["decode"] = "keep values (mwdg2_set_decode_mode 1)"
    return out


def run_learned(a):
    """The learned refinement proposal on the 4096^2 catchment: the same
    case run from t = 0 to --eval-time on this GPU -- plain in FP64 (the depth reference),
    then in --precision plain, with the trained MLP proposing the subtrees the encode and
    decode visit (a full judge step every --judge-every steps), and both again with the
    keep-values decode (mwdg2_set_decode_mode 1). Each run's device time is the sum of its
    steps' CUDA-event times (input resident, no host copies); the depth error is the largest
    difference, over every finest cell, of the depth at the cell centre from the FP64 run's
    at the same simulated time (each run ends exactly at --eval-time). Prints one line per
    run in --precision."""
    import numpy as np
    import torch
    import cases
    import mwdg2_b200
    torch.cuda.set_device(0)
    base = a.case_dir or os.path.join(tempfile.gettempdir(), "mwdg2_bench_cases")
    d = os.path.join(base, f"learned-{a.level}-{a.eval_time:g}-v1")
    par = os.path.join(d, "case.par")
    if not os.path.exists(os.path.join(d, "READY")):
        os.makedirs(d, exist_ok=True)
        cases.fbm_catchment(d, L=a.level, sim_time=a.eval_time)
        open(os.path.join(d, "READY"), "w").close()
    z = np.load(a.proposal)
    params = z["params"]
    train = json.loads(str(z["summary"]))

    def run(precision, learned, keep=False):
        sim = mwdg2_b200.Simulation(par, precision=precision, timing="step")
        if keep:
            sim.set_decode_mode("keep")
        if learned:
            sim.proposal_enable(params, judge_every=a.judge_every, threshold=train["threshold"], miss_bound=0.02)
        ms, leaves, steps, applied = 0.0, 0, 0, 0
        while True:
            ok, dt, n = sim.step()
            if not ok:
                break
            ms += float(sim.last_step_timing()[7])
            leaves += n
            steps += 1
            if learned:
                applied += int(sim.proposal_stats()["applied"])
        out = {"ms": ms, "leaves": leaves, "steps": steps, "time": sim.info()["time"], "depth": finest_depth(sim),
               "wet_volume": wet_volume(sim)}
        if learned:
            out["stats"] = sim.proposal_stats()
            out["applied_steps"] = applied
        sim.close()
        return out

    # the plain FP64 run is the depth reference; plain and learned run in --precision
    ref = run(64, False)
    plain = ref if a.precision == 64 else run(a.precision, False)
    runs = (("plain", plain), ("learned", run(a.precision, True)), ("keep", run(a.precision, False, keep=True)),
            ("learned+keep", run(a.precision, True, keep=True)))
    fp = f"FP{a.precision}"
    lines = []
    for name, r in runs:
        err = float(np.max(np.abs(r["depth"] - ref["depth"])))
        line = {"metric": METRIC + f" ({name} {fp} vs plain FP64 depth)", "value": r["leaves"] / (r["ms"] / 1e3),
                "unit": UNIT, "n_gpus": 1, "steps": r["steps"], "warmup": 0, "ms_per_step": r["ms"] / r["steps"],
                "higher_is_better": True, "impl": f"ours-{name}", "dtype": f"f{a.precision}",
                "data": "synthetic (seeded fBm DEM, no network)",
                "config": {"workload": f"fBm catchment {1 << a.level}^2 (max_ref_lvl {a.level}) run from t = 0 to "
                                       f"{a.eval_time:g} s (the hydrograph peak), MWDG2 {fp}",
                           "proposal": "none" if "learned" not in name else
                                       f"trained MLP ({a.proposal.split('/')[-1]}), judge every {a.judge_every} steps",
                           "decode": "keep values" if "keep" in name else "reference",
                           "depth_reference": "the same case in FP64, plain"},
                "max_depth_error_m": err, "time": r["time"], "reference_time": ref["time"],
                "wet_volume_m3": r["wet_volume"], "reference_wet_volume_m3": ref["wet_volume"],
                "timing": "sum of CUDA-event device times of every step of the run"}
        if name != "plain":
            line["vs_plain"] = line["value"] / lines[0]["value"]
        if "learned" in name:
            line["proposal"] = {**r["stats"], "applied_steps": r["applied_steps"], "training": train}
        lines.append(line)
    for line in lines:
        print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload == "ensemble":
        run_ensemble(a)
        return
    if a.workload == "learned":
        run_learned(a)
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
    t_init = time.perf_counter()
    # step timing: two events around each step's device work, outside its captured graph
    sim = mwdg2_b200.Simulation(par, precision=a.precision, device=local, timing="step")
    sim.set_decode_mode(a.decode)
    t_init = time.perf_counter() - t_init   # reading the rasters + device initialisation
    clk = Clocks(local).__enter__()   # sampled from the warm-up through the end-to-end loop
    for _ in range(a.warmup):
        sim.step()

    # device-timed steps (replicas: every rank runs the same workload on its own GPU)
    barrier()
    t_sim0 = sim.info()["time"]
    ms_step, leaves, counters = [], [], []
    with nvtx_range("timed_window"):
        for _ in range(a.steps):
            ok, dt, n = sim.step()
            ms_step.append(float(sim.last_step_timing()[7]))
            leaves.append(n)
            counters.append(sim.last_step_counters())
    barrier()
    sim_s = sim.info()["time"] - t_sim0
    tot_ms = max_over_ranks(float(sum(ms_step)), dist, "cuda")
    value = replica_throughput(world, sum(leaves), tot_ms)
    # phase breakdown (and the dominant phase's time for the roofline), right after the timed
    # steps: a separate pass with events between the phases inside the step's graph, which
    # the timed steps do not carry (each such event node costs ~10 us of launch pipelining);
    # its first step captures the graph variant with the events and is not used
    sim.set_timing("phases")
    sim.step()
    ms_phase, leaves_ph = [], []
    for _ in range(PHASE_STEPS):
        ok, dt, n = sim.step()
        ms_phase.append(sim.last_step_timing().tolist())
        leaves_ph.append(n)
    sim.set_timing("step")
    barrier()

    learned = None
    want_learned = world == 1 and a.workload == "catchment" and a.solver == "mwdg2" and os.path.exists(a.proposal)
    keep = None
    if want_learned:
        learned = learned_window(a, par, 0.0, sim.info()["time"], finest_depth(sim), value, "learned_window",
                                 wet_volume(sim))
    if world == 1 and a.workload == "catchment" and a.decode == "reference":
        keep = learned_window(a, par, 0.0, sim.info()["time"], finest_depth(sim), value, "keep_window",
                              wet_volume(sim), mode="keep")

    # end to end through the C ABI: the library's own time loop (mwdg2_run) over K steps; each
    # step's dt, boundary and point-source values go host->device from pinned memory, and its
    # scalars with the stage-point values come back device->host in one copy, which the host
    # waits for before the next step
    barrier()
    t0 = time.perf_counter()
    e2e_steps, e2e_leaves = sim.run(a.steps)
    barrier()
    e2e_wall = time.perf_counter() - t0
    clk.__exit__(None, None, None)
    e2e_wall = max_over_ranks(e2e_wall, dist, "cuda")
    P = a.precision // 8
    # bytes the library copied per step (its counters): host->device the step's dt, boundary
    # and point-source values; device->host its scalars and the stage-point values
    h2d = int(counters[-1]["h2d_bytes"])
    d2h = int(counters[-1]["d2h_bytes"])

    # roofline of the dominant kernel, from its live event timing
    ph = np.array(ms_phase)
    mean_ph = ph.mean(axis=0)
    n_mean = float(np.mean(leaves))
    n_mean_ph = float(np.mean(leaves_ph))
    peak, peak_kind = peaks()
    # Per-leaf algorithmic bytes of the reference-layout model: leaf topology 40 B (code,
    # level, 4 x (neighbour id, level)); RK stage 1: 12P own coefficients + 16 B neighbour
    # ids + 9P written + 9P of U^n = 30P + 16; stage 2: 21P + 16 (together the N(51P + 32)
    # solver term of the step formula below). HWFV1: 4P own + 16 B ids + 3P written.
    cand = {"leaf topology (k_tile_count + k_tile_scan + k_tile_emit)": (3, 40),
            "RK stage 1 (k_stage_wet<1>, then k_stage_dry<1> beside k_mwdg2_stage<1> over the wet list; or "
            "one k_mwdg2_stage<1> sweep)": (4, 30 * P + 16),
            "RK stage 2 (k_stage_wet<2>, then k_stage_dry<2> beside k_mwdg2_stage<2> over the wet list; or "
            "one k_mwdg2_stage<2> sweep)": (6, 21 * P + 16)}
    if a.solver == "hwfv1":
        cand = {"leaf topology (k_tile_count + k_tile_scan + k_tile_emit)": (3, 40),
                "k_hwfv1 (gather, friction, FV1 update, CFL)": (4, 7 * P + 16)}
    kname, (kph, per_leaf) = max(cand.items(), key=lambda kv: mean_ph[kv[1][0]])
    kms = float(mean_ph[kph])
    traffic = TRAFFIC_B_PER_LEAF.get((a.solver, P, kph)) if (a.workload, a.level) == ("catchment", 12) else None
    achieved = per_leaf * n_mean_ph / (kms / 1e3) / 1e9
    # Algorithmic bytes per step of the reference-layout model, from each step's device
    # counters: E parents encoded, E2 re-encoded (scale only), D decoded, T detail slots,
    # N leaves; MWDG2 B = E(73P+1) + E2*45P + T(P+2) + D*72P + 40N + N(51P+32), HWFV1
    # B = E(25P+1) + T(P+2) + D*24P + 40N + N(7P+16). This build stores no details or norms,
    # so its encode moves fewer bytes than the model counts.
    if a.solver == "mwdg2":
        formula = "E(73P+1)+E2*45P+T(P+2)+D*72P+40N+N(51P+32)"
        per_step = [c["encoded"] * (73 * P + 1) + c["reencoded"] * 45 * P + c["detail_slots"] * (P + 2) +
                    c["decoded"] * 72 * P + 40 * c["leaves"] + c["leaves"] * (51 * P + 32) for c in counters]
    else:
        formula = "E(25P+1)+T(P+2)+D*24P+40N+N(7P+16)"
        per_step = [c["encoded"] * (25 * P + 1) + c["detail_slots"] * (P + 2) + c["decoded"] * 24 * P +
                    40 * c["leaves"] + c["leaves"] * (7 * P + 16) for c in counters]
    step_bytes = float(np.mean(per_step))
    step_gbs = step_bytes / (statistics.mean(ms_step) / 1e3) / 1e9

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": tot_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"f{a.precision}", "data": "synthetic (seeded fBm DEM, no network)", "config": workload(a),
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic * n_mean_ph if traffic else None,
                         "traffic_source": TRAFFIC_SOURCE if traffic else None,
                         "bytes_per_leaf": per_leaf, "leaves_per_launch": n_mean_ph, "kernel_ms": kms},
            "roofline_step": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_gbs, "frac": step_gbs / peak,
                              "formula": formula},
            "e2e": {"value": world * e2e_leaves / e2e_wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "timing": "host clock around mwdg2_run over K steps (the library's time loop)"},
            "gpu_launches": int(sum(cc["launches"] for cc in counters)),
            "clocks": clk.summary(),
            "phase_ms_mean": dict(zip(("step_open", "encode", "decode", "topology", "stage1",
                                       "reencode", "stage2", "step"), [round(x, 4) for x in mean_ph])),
            "phase_timing": f"{PHASE_STEPS} steps after the timed ones with events between the phases inside "
                            "the step's graph (the timed steps carry none; each adds ~10 us)",
            "leaves_mean": n_mean,
            "wall_s_per_sim_s": {"value": (tot_ms / 1e3) / sim_s if sim_s > 0 else None, "sim_seconds": sim_s,
                                 "window": f"steps {a.warmup + 1}..{a.warmup + a.steps} of the run (device time of "
                                           "the timed steps over the simulated time they advanced)"},
            "init_s": t_init,
            "wet_fraction": [float(np.mean([cc[k] for cc in counters])) / n_mean for k in ("wet_stage1", "wet_stage2")]}
    if learned is not None:
        line["learned"] = learned
    if keep is not None:
        line["decode_keep"] = keep
    if a.workload == "catchment" and a.peak_time > 0:
        wp = peak_window(sim, a, dist)
        t_end, depth_end = wp.pop("_end_time", None), wp.pop("_end_depth", None)
        line["window_peak"] = wp
        if want_learned and "value" in wp:
            wp["learned"] = learned_window(a, par, a.peak_time, t_end, depth_end, wp["value"], "learned_peak_window",
                                           wp["wet_volume_m3"])
        if keep is not None and "value" in wp:
            wp["decode_keep"] = learned_window(a, par, a.peak_time, t_end, depth_end, wp["value"], "keep_peak_window",
                                               wp["wet_volume_m3"], mode="keep")
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
