"""Water volume of the reference's own CUDA build after a given step (test infrastructure).

Runs the reference build (oracle/_ref/gpu-mwdg2-ref-fp{32,64}, the reference's unmodified
sources with the observation wrappers of oracle/ref/hooks.cu) on a case until it has
finished step `step`, has the wrappers dump its leaf state after that step
(MWDG2_REF_DUMP_DIR / MWDG2_REF_DUMP_STEPS: the arrays `levels` and `h0` of its assembled
solution), and returns the water volume in the leaves at least `tol_h` deep, the fraction
of leaves that deep and the simulated time of the step. Used to compare the long-run water
of this build's FP32 and FP64 runs with the reference's.

    python oracle/reference_wet_volume.py <case.par> <precision> <step> [dx] [max_ref_lvl]
"""
import csv
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_wet_volume(par: str, precision: int, step: int, dx: float, L: int, tol_h: float = 1e-3,
                         exe: str | None = None, timeout: float = 1800.0) -> dict:
    work = os.path.dirname(os.path.abspath(par))
    exe = os.path.abspath(exe) if exe else os.path.join(HERE, "_ref", f"gpu-mwdg2-ref-fp{precision}")
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} is missing: build it with `make -C oracle ref`")
    with tempfile.TemporaryDirectory() as dump:
        log = os.path.join(dump, "steps.csv")
        # the state after step k is dumped at the start of step k + 1
        env = dict(os.environ, MWDG2_REF_DUMP_DIR=dump, MWDG2_REF_DUMP_STEPS=str(step),
                   MWDG2_REF_STOP_AFTER=str(step + 1), MWDG2_REF_STEPS_CSV=log)
        r = subprocess.run([exe, os.path.basename(par)], cwd=work, env=env, capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference build exited {r.returncode}: {r.stderr[-2000:]}")
        rows = list(csv.DictReader(open(log)))
        real = np.float32 if precision == 32 else np.float64
        lvl = np.fromfile(os.path.join(dump, f"step{step:06d}_levels.bin"), dtype=np.int32).astype(np.int64)
        h = np.fromfile(os.path.join(dump, f"step{step:06d}_h0.bin"), dtype=real).astype(np.float64)
    area = dx * dx * np.ldexp(1.0, 2 * (L - lvl))
    wet = h >= tol_h
    return {"precision": precision, "step": step, "time": float(rows[step - 1]["time"]), "leaves": int(h.size),
            "wet_volume_m3": float(np.sum(np.where(wet, h, 0.0) * area)), "wet_fraction": float(np.mean(wet))}


if __name__ == "__main__":
    a = sys.argv[1:]
    print(json.dumps(reference_wet_volume(a[0], int(a[1]), int(a[2]), float(a[3]) if len(a) > 3 else 2.0,
                                          int(a[4]) if len(a) > 4 else 12)))
