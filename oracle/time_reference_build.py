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
                              case_dir=a.case_dir)
    par = bench.make_case(case, 0)
    work = os.path.dirname(os.path.abspath(par))
    exe = os.path.abspath(a.exe) if a.exe else os.path.join(HERE, "_ref", f"gpu-mwdg2-ref-fp{a.precision}")
    if not os.path.exists(exe):
        raise SystemExit(f"{exe} is missing: build it with `make -C oracle ref`")
    log = os.path.join(work, f"ref_steps_{a.solver}_fp{a.precision}.csv")
    env = dict(os.environ, MWDG2_REF_STOP_AFTER=str(a.warmup + a.steps), MWDG2_REF_STEPS_CSV=log)
    r = subprocess.run([exe, os.path.basename(par)], cwd=work, env=env, capture_output=True, text=True,
                       timeout=1800)
    if r.returncode != 0:
        raise SystemExit(f"reference build exited {r.returncode}: {r.stderr[-2000:]}")
    rows = list(csv.DictReader(open(log)))
    if len(rows) < a.warmup + a.steps:
        raise SystemExit(f"reference build logged {len(rows)} steps, {a.warmup + a.steps} wanted")
    t0 = float(rows[a.warmup - 1]["wall_s"]) if a.warmup > 0 else 0.0
    t1 = float(rows[a.warmup + a.steps - 1]["wall_s"])
    leaves = sum(int(rw["n_leaves"]) for rw in rows[a.warmup:a.warmup + a.steps])
    print(json.dumps({"impl": "reference CUDA build", "solver": a.solver, "dtype": f"f{a.precision}",
                      "workload": bench.workload(case)["workload"], "steps": a.steps, "warmup": a.warmup,
                      "ms_per_step": 1e3 * (t1 - t0) / a.steps, "value": leaves / (t1 - t0),
                      "unit": "cell-updates/s", "leaves_mean": leaves / a.steps,
                      "timing": "host wall clock between the ends of steps W and W+K (each step ends with a "
                                "device-to-host copy of dt)"}), flush=True)


if __name__ == "__main__":
    main()
