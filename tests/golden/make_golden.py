"""Generate golden fixtures by running the reference implementation.

Runs the reference build (oracle/_ref/gpu-mwdg2-ref-fp{64,32}, made by
`make -C oracle ref` from the al0vya/gpu-mwdg2 sources) on small seeded cases and packs
what its observation hooks dump (oracle/ref/hooks.cu) into compressed .npz files:

  per dumped step n:  leaf list (act_idcs, levels), neighbour ids/levels, significance
                      flags, dt, maxes, and the leaf state after step n.

The reference only runs on a GPU, so this script is run on a machine with one:

    python tests/golden/make_golden.py --out <dir>

and the resulting files are copied into tests/golden/. Tests then use them to pin the
CPU oracle and the CUDA product. Inputs are regenerated from the same seeds, so the
fixtures hold outputs only.
"""
from __future__ import annotations

import argparse
import glob
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

DUMP_STEPS = (1, 2, 3, 10, 40)


def case_specs():
    """Name -> (generator kwargs, precision). Kept small: fixtures are committed."""
    specs = {
        "cdb_mw_l7_fp64": (dict(kind="cdb", L=7, solver="mwdg2"), 64),
        "cdb_mw_l7_fp32": (dict(kind="cdb", L=7, solver="mwdg2"), 32),
        "cdb_hw_l7_fp64": (dict(kind="cdb", L=7, solver="hwfv1"), 64),
        "fbm_mw_l7_fp64": (dict(kind="fbm", L=7, solver="mwdg2"), 64),
        "fbm_hw_l7_fp64": (dict(kind="fbm", L=7, solver="hwfv1"), 64),
        "lake_mw_l7_fp64": (dict(kind="lake", L=7, solver="mwdg2"), 64),
        # boundary segments of every type on the four sides (two layouts)
        "edges_a_mw_l7_fp64": (dict(kind="edges_a", L=7, solver="mwdg2"), 64),
        "edges_a_hw_l7_fp64": (dict(kind="edges_a", L=7, solver="hwfv1"), 64),
        "edges_b_mw_l7_fp64": (dict(kind="edges_b", L=7, solver="mwdg2"), 64),
        "edges_b_hw_l7_fp64": (dict(kind="edges_b", L=7, solver="hwfv1"), 64),
        "edges_a_mw_l7_fp32": (dict(kind="edges_a", L=7, solver="mwdg2"), 32),
        # a 120 x 100 DEM with no-data cells, initial discharge from .start.Qx/.Qy
        "startq_mw_l7_fp64": (dict(kind="startq", L=7, solver="mwdg2"), 64),
        "startq_hw_l7_fp64": (dict(kind="startq", L=7, solver="hwfv1"), 64),
    }
    return specs


def make_case(kind: str, directory: str, L: int, solver: str):
    if kind == "cdb":
        return cases.circular_dam_break(directory, L=L, solver=solver, sim_time=3.5, massint=None)
    if kind == "fbm":
        n = 1 << L
        z = cases.fbm_surface(n, 0.8, 20261203, 30.0)
        h0 = np.maximum(0.0, 12.0 - z)
        return cases.fbm_catchment(directory, L=L, solver=solver, cellsize=2.0, sim_time=600.0,
                                   manning=0.03, peak_q=50.0, t_peak=300.0, start_depth=h0,
                                   limitslopes=(solver == "mwdg2"))
    if kind == "lake":
        return cases.lake_at_rest(directory, L=L, solver=solver, sim_time=10.0)
    if kind in ("edges_a", "edges_b"):
        return cases.bc_edges(directory, variant=kind[-1], L=L, solver=solver)
    if kind == "startq":
        return cases.start_q_nodata(directory, L=L, solver=solver)
    raise ValueError(kind)


def read_dump(d: str, step: int, name: str, dtype):
    path = os.path.join(d, f"step{step:06d}_{name}.bin")
    if not os.path.exists(path):
        return None
    return np.fromfile(path, dtype=dtype)


STATE_SAMPLE = 1024


def trim(arrays: dict) -> dict:
    """Keep fixtures small: topology, flags and dt are kept whole; leaf-state arrays
    longer than 2*STATE_SAMPLE are reduced to a fixed random sample of leaves
    (indices stored as sN_state_idx) plus float64 sums of every state array."""
    out = {}
    rng = np.random.Generator(np.random.PCG64(0))
    for k, v in arrays.items():
        if "_state_" in k and not k.endswith(("_len", "_act", "_lvl", "_idx", "_sum")):
            step = k.split("_")[0]
            n = v.shape[0]
            out[f"{k}_sum"] = np.array([np.sum(v.astype(np.float64))])
            if n > 2 * STATE_SAMPLE:
                ik = f"{step}_state_idx"
                if ik not in out:
                    out[ik] = np.sort(rng.choice(n, STATE_SAMPLE, replace=False)).astype(np.int32)
                v = v[out[ik]]
            out[k] = v
        elif k.endswith("_norm"):
            continue  # norms are only kept implicitly through the significance flags
        else:
            out[k] = v
    # state act/lvl are the leaf list of the previous step's compaction; keep sampled too
    for k in list(out):
        if k.endswith(("_state_act", "_state_lvl")):
            ik = k.split("_")[0] + "_state_idx"
            if ik in out:
                out[k] = out[k][out[ik]]
    return out


def run_case(name: str, spec, ref_dir: str, out_dir: str, max_step: int) -> dict:
    kw, prec = spec
    work = tempfile.mkdtemp(prefix="golden_")
    c = make_case(kw["kind"], work, kw["L"], kw["solver"])
    dump = os.path.join(work, "dump")
    os.makedirs(dump)
    exe = os.path.join(ref_dir, f"gpu-mwdg2-ref-fp{prec}")
    env = dict(os.environ, MWDG2_REF_DUMP_DIR=dump,
               MWDG2_REF_DUMP_STEPS=",".join(str(s) for s in DUMP_STEPS),
               MWDG2_REF_STOP_AFTER=str(max_step + 1),
               MWDG2_REF_STEPS_CSV=os.path.join(work, "steps.csv"))
    r = subprocess.run([exe, os.path.basename(c.par)], cwd=work, env=env, capture_output=True,
                       text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}: {r.stderr[-2000:]}")
    real = np.float64 if prec == 64 else np.float32
    arrays = {}
    for s in DUMP_STEPS:
        if s > max_step:
            continue
        pre = f"s{s}_"
        n = read_dump(dump, s, "leaf_len", np.int32)
        if n is None:
            continue
        arrays[pre + "leaf_act"] = read_dump(dump, s, "leaf_act_idcs", np.int32)
        arrays[pre + "leaf_lvl"] = read_dump(dump, s, "leaf_levels", np.int32)
        for d in "nesw":
            arrays[pre + f"nb_{d}_ids"] = read_dump(dump, s, f"nb_{d}_ids", np.int32)
            lv = read_dump(dump, s, f"nb_{d}_lvls", np.int32)
            if lv is not None:
                arrays[pre + f"nb_{d}_lvls"] = lv
        arrays[pre + "sig"] = read_dump(dump, s, "sig", np.uint8)
        arrays[pre + "norm"] = read_dump(dump, s, "norm", real)
        arrays[pre + "dt"] = read_dump(dump, s, "dt", real)
        arrays[pre + "maxes"] = read_dump(dump, s, "maxes", real)
        for f in ("h0", "qx0", "qy0", "z0", "h1x", "qx1x", "qy1x", "z1x", "h1y", "qx1y", "qy1y", "z1y"):
            a = read_dump(dump, s, f, real)
            if a is not None:
                arrays[pre + "state_" + f] = a
        sn = read_dump(dump, s, "len", np.int32)
        if sn is not None:
            arrays[pre + "state_len"] = sn
            arrays[pre + "state_act"] = read_dump(dump, s, "act_idcs", np.int32)
            arrays[pre + "state_lvl"] = read_dump(dump, s, "levels", np.int32)
    arrays = {k: v for k, v in arrays.items() if v is not None}
    steps = np.genfromtxt(os.path.join(work, "steps.csv"), delimiter=",", names=True)
    arrays["steps_dt"] = np.atleast_1d(steps["dt"]).astype(np.float64)
    arrays["steps_n"] = np.atleast_1d(steps["n_leaves"]).astype(np.int64)
    out = os.path.join(out_dir, f"{name}.npz")
    np.savez_compressed(out, **trim(arrays))
    shutil.rmtree(work, ignore_errors=True)
    return {"name": name, "case": kw, "precision": prec, "steps": int(len(arrays["steps_dt"])),
            "bytes": os.path.getsize(out)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--retrim", default=None, help="re-trim untrimmed .npz files in this directory")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--ref-dir", default=os.path.join(ROOT, "oracle", "_ref"))
    ap.add_argument("--max-step", type=int, default=40)
    ap.add_argument("--only", default=None)
    ap.add_argument("--append", action="store_true", help="keep the other entries of index.json")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.retrim:
        for f in sorted(glob.glob(os.path.join(a.retrim, "*.npz"))):
            z = dict(np.load(f))
            dst = os.path.join(a.out, os.path.basename(f))
            np.savez_compressed(dst, **trim(z))
            print(os.path.basename(f), os.path.getsize(dst))
        idx = os.path.join(a.retrim, "index.json")
        if os.path.exists(idx):
            shutil.copy(idx, os.path.join(a.out, "index.json"))
        return
    index_path = os.path.join(a.out, "index.json")
    index = json.load(open(index_path)) if a.append and os.path.exists(index_path) else []
    for name, spec in case_specs().items():
        if a.only and not any(o in name for o in a.only.split(",")):
            continue
        info = run_case(name, spec, a.ref_dir, a.out, a.max_step)
        print(json.dumps(info), flush=True)
        index = [e for e in index if e["name"] != name] + [info]
    with open(os.path.join(a.out, "index.json"), "w") as fp:
        json.dump(index, fp, indent=1)


if __name__ == "__main__":
    main()
