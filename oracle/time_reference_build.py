"""Times the reference's own CUDA build on the benchmark case (measurement infrastructure).

Runs oracle/_ref/gpu-mwdg2-ref-fp{32,64} (made by `make -C oracle ref` from the reference
sources; the oracle/ref/hooks.cu wrappers log each step's leaf count and wall time after
the reference's get_dt_CFL, run_simulation.cu:650, which ends every step with a
device-to-host copy) on the case bench.py builds for the same arguments, stops it after
W + K steps and prints one JSON line: ms per step and active-cell updates/s over steps
W+1..W+K (leaves of those steps / wall time between the end of step W and of step W+K).

  python oracle/time_reference_build.py [--precision 32|64] [--solver mwdg2|hwfv1]
                                        [--level 12] [--steps 20] [--warmup 3]
"""
from __future__ import annotations

import argparse
import csv
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def time_reference(par: str, precision: int, steps: int, warmup: int, exe: str | None = None,
                   timeout: float = 1800.0, window_time: float | None = None) -> dict:
    """Runs the reference build on `par` (from its folder) and times `steps` steps after
    `warmup` untimed ones, from its per-step log: ms per step, active-cell updates/s and
    wall seconds per simulated second (the simulated time of a step is the dt the step
    before it logged). The window starts at the beginning of the run, or with
    `window_time` after the first step that ends at or after that simulated time."""
    work = os.path.dirname(os.path.abspath(par))
    exe = os.path.abspath(exe) if exe else os.path.join(HERE, "_ref", f"gpu-mwdg2-ref-fp{precision}")
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} is missing: build it with `make -C oracle ref`")
    log = os.path.join(work, f"ref_steps_{os.getpid()}.csv")
    env = dict(os.environ, MWDG2_REF_STEPS_CSV=log)
    if window_time is None:
        env["MWDG2_REF_STOP_AFTER"] = str(warmup + steps)
    else:
        env["MWDG2_REF_WINDOW_TIME"] = repr(float(window_time))
        env["MWDG2_REF_WINDOW_STEPS"] = str(warmup + steps)
    r = subprocess.run([exe, os.path.basename(par)], cwd=work, env=env, capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference build exited {r.returncode}: {r.stderr[-2000:]}")
    rows = list(csv.DictReader(open(log)))
    os.remove(log)
    first = 0   # rows before the window (row k - 1 is step k)
    if window_time is not None:
        hits = [k for k, rw in enumerate(rows) if float(rw.get("time", "-1")) >= window_time]
        if not hits:
            raise RuntimeError(f"reference build never reached t = {window_time} s")
        first = hits[0] + 1
    if len(rows) < first + warmup + steps:
        raise RuntimeError(f"reference build logged {len(rows)} steps, {first + warmup + steps} wanted")
    w0 = first + warmup
    t0 = float(rows[w0 - 1]["wall_s"]) if w0 > 0 else 0.0
    t1 = float(rows[w0 + steps - 1]["wall_s"])
    leaves = sum(int(rw["n_leaves"]) for rw in rows[w0:w0 + steps])
    # step k advances the clock by the dt logged at the end of step k - 1
    sim = sum(float(rw["dt"]) for rw in rows[max(0, w0 - 1):w0 + steps - 1])
    out = {"impl": "reference CUDA build", "dtype": f"f{precision}", "steps": steps, "warmup": warmup,
           "ms_per_step": 1e3 * (t1 - t0) / steps, "value": leaves / (t1 - t0), "unit": "cell-updates/s",
           "leaves_mean": leaves / steps, "sim_seconds": sim,
           "wall_s_per_sim_s": (t1 - t0) / sim if sim > 0 else None,
           "timing": "host wall clock between the ends of steps W and W+K of the window (each step ends with "
                     "a device-to-host copy of dt)"}
    if window_time is not None:
        out["window"] = {"from_time": window_time, "first_step": w0 + 1,
                         "time": float(rows[w0]["time"]) if "time" in rows[w0] else None}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--solver", default="mwdg2", choices=["mwdg2", "hwfv1"])
    ap.add_argument("--level", type=int, default=12)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--case-dir", default=None)
    ap.add_argument("--exe", default=None, help="reference executable (default: oracle/_ref/gpu-mwdg2-ref-fp<P>)")
    a = ap.parse_args()
    sys.path.insert(0, ROOT)
    import bench
    case = argparse.Namespace(workload="catchment", level=a.level, solver=a.solver, precision=a.precision,
                              case_dir=a.case_dir, window="start")
    par = bench.make_case(case, 0)
    try:
        d = time_reference(par, a.precision, a.steps, a.warmup, a.exe)
    except (FileNotFoundError, RuntimeError) as e:
        raise SystemExit(str(e))
    d.update({"solver": a.solver, "workload": bench.workload(case)["workload"]})
    print(json.dumps(d), flush=True)


if __name__ == "__main__":
    main()
