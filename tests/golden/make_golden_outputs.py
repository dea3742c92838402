"""Golden output files (saveint raster maps, VTK, c-prop CSVs, res.cumu) from the reference.

Runs the reference build (oracle/_ref/gpu-mwdg2-ref-fp{64,32}, made by `make -C oracle ref`
from the al0vya/gpu-mwdg2 sources) through its own run_simulation on small seeded dam
breaks whose .par files switch on the saveint outputs, and stores every file it writes as
raw text in one compressed .npz per case (key = path relative to the case directory).
The reference only runs on a GPU, so this script is run on a machine with one:

    python tests/golden/make_golden_outputs.py --out <dir>

and the resulting files are copied into tests/golden/. Inputs are regenerated from the
same generator arguments, so the fixtures hold outputs only.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu-mwdg2_b200"))
import cases  # noqa: E402


def output_specs():
    """Name -> (kind, solver, max_ref_lvl, precision, output keywords). Kept small: committed."""
    return {
        "out_cdb_mw_l6_fp64": ("cdb", "mwdg2", 6, 64, ["raster_out", "vtk", "c_prop", "voutput", "qoutput"]),
        "out_cdb_hw_l6_fp64": ("cdb", "hwfv1", 6, 64, ["raster_out", "vtk", "c_prop", "qoutput"]),
        "out_cdb_mw_l6_fp32": ("cdb", "mwdg2", 6, 32, ["raster_out", "voutput", "c_prop"]),
        "out_fbm_mw_l6_fp64": ("fbm", "mwdg2", 6, 64, ["raster_out", "vtk", "voutput"]),
    }


def make_output_case(directory: str, kind: str, solver: str, L: int, keywords: list[str]):
    """Two saves (the first step, and t >= 0.25 s of a dam break or t >= 2 s of a catchment
    with standing water over an fBm bed and a point inflow: some 10 and 40 steps) of the
    requested outputs."""
    if kind == "cdb":
        return cases.circular_dam_break(directory, L=L, solver=solver, sim_time=0.3, massint=None,
                                        saveint=0.25, extra=keywords)
    n = 1 << L
    z = cases.fbm_surface(n, 0.8, 20261203, 30.0)
    return cases.fbm_catchment(directory, L=L, solver=solver, cellsize=2.0, sim_time=2.5, manning=0.03,
                               peak_q=50.0, t_peak=300.0, start_depth=np.maximum(0.0, 12.0 - z),
                               limitslopes=True, massint=None, saveint=2.0, extra=keywords)


def collect_outputs(work: str) -> dict[str, str]:
    """Every file the run wrote: the dirroot folder `res/` and the c-prop CSVs, which the
    reference names <dirroot><name>.csv next to the .par."""
    out = {}
    for root, _, files in os.walk(work):
        for f in files:
            p = os.path.join(root, f)
            rel = os.path.relpath(p, work)
            if rel.startswith("res"):   # the case's inputs are named case.*
                with open(p) as fp:
                    out[rel] = fp.read()
    return out


def run_case(name: str, spec, ref_dir: str, out_dir: str) -> dict:
    kind, solver, L, prec, kws = spec
    work = tempfile.mkdtemp(prefix="golden_out_")
    c = make_output_case(work, kind, solver, L, kws)
    exe = os.path.join(ref_dir, f"gpu-mwdg2-ref-fp{prec}")
    r = subprocess.run([exe, os.path.basename(c.par)], cwd=work, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}: {r.stderr[-2000:]}")
    files = collect_outputs(work)
    arrays = {k: np.frombuffer(v.encode(), dtype=np.uint8) for k, v in files.items()}
    out = os.path.join(out_dir, f"{name}.npz")
    np.savez_compressed(out, **arrays)
    shutil.rmtree(work, ignore_errors=True)
    return {"name": name, "files": sorted(files), "bytes": os.path.getsize(out)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--ref-dir", default=os.path.join(ROOT, "oracle", "_ref"))
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    index = [run_case(n, s, a.ref_dir, a.out) for n, s in output_specs().items()]
    for i in index:
        print(json.dumps(i), flush=True)
    with open(os.path.join(a.out, "outputs_index.json"), "w") as fp:
        json.dump(index, fp, indent=1)


if __name__ == "__main__":
    main()
