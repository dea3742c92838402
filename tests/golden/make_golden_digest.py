"""Generate per-step digest fixtures by running the reference implementation.

For runs too large to store whole (the 4096^2 benchmark catchment at max_ref_lvl 12) or
too long (the 256^2 circular dam break over its full 3.5 s), the reference build
(oracle/_ref/gpu-mwdg2-ref-fp{64,32}, made by `make -C oracle ref` from the al0vya/gpu-mwdg2
sources) writes, through its observation hooks (oracle/ref/hooks.cu, MWDG2_REF_DIGEST_DIR):

  every step:          a 64-bit digest of the leaf list (hierarchy indices, levels), the
                       four neighbour id arrays (and, MWDG2, their levels) and the
                       significance flags, plus dt and the leaf count;
  at a few steps:      the leaf state at up to 2048 evenly spaced leaves (index j*n/S)
                       and the float64 sums of the 12 state rows.

This script packs them into tests/golden/digest_<name>.npz. The reference only runs on a
GPU, so it is run on a machine with one:

    python tests/golden/make_golden_digest.py [--only NAME] [--out DIR]

Inputs are regenerated from the case generators' seeds, so the fixtures hold outputs only.
`digest()` is the same function as the hooks' (numpy, wrapping uint64 arithmetic); the
tests use it on the product's arrays.
"""
from __future__ import annotations

import argparse
import csv
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

SAMPLE = 2048
TOPOLOGY = ("leaf_act", "leaf_lvl", "nb_n_ids", "nb_e_ids", "nb_s_ids", "nb_w_ids",
            "nb_n_lvls", "nb_e_lvls", "nb_s_lvls", "nb_w_lvls")
NAMES = TOPOLOGY + ("sig",)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """Vigna's splitmix64 finaliser of x + 0x9E3779B97F4A7C15, elementwise (uint64, wrapping)."""
    x = x.astype(np.uint64) + _GOLDEN
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


class Digester:
    """digest(a) = n * 0x9E3779B97F4A7C15 + sum_i (bits(a_i) + 1) * (splitmix64(i) | 1) mod 2^64,
    bits() the 8- or 32-bit pattern of the value, zero-extended. Multipliers are cached."""

    def __init__(self):
        self._m = np.zeros(0, np.uint64)

    def _mult(self, n: int) -> np.ndarray:
        if self._m.size < n:
            self._m = _splitmix64(np.arange(max(n, 2 * self._m.size), dtype=np.uint64)) | np.uint64(1)
        return self._m[:n]

    def __call__(self, a: np.ndarray, bits: int = 32) -> int:
        a = np.ascontiguousarray(a)
        n = a.size
        if bits == 32:
            v = a.astype(np.int64).astype(np.uint32) if a.dtype.itemsize != 4 else a.view(np.uint32)
        else:
            v = a.astype(np.uint8)
        with np.errstate(over="ignore"):
            s = np.sum((v.astype(np.uint64) + np.uint64(1)) * self._mult(n), dtype=np.uint64)
            return int((np.uint64(n) * _GOLDEN + s) & np.uint64(0xFFFFFFFFFFFFFFFF))


def case_specs() -> dict:
    """Name -> spec. `steps`: steps compared (None: the whole run); `samples`: steps whose
    sampled state is kept."""
    cat = dict(kind="catchment", L=12, steps=25, samples=(1, 5, 12, 25))
    full = dict(kind="cdb", L=8, steps=None, samples=(1, 50, 100, 150, 200, 250, 290))
    return {
        "catch_mw_l12_fp32": dict(cat, solver="mwdg2", precision=32),
        "catch_mw_l12_fp64": dict(cat, solver="mwdg2", precision=64),
        "catch_hw_l12_fp32": dict(cat, solver="hwfv1", precision=32),
        "catch_hw_l12_fp64": dict(cat, solver="hwfv1", precision=64),
        "cdb_mw_l8_fp64_full": dict(full, solver="mwdg2", precision=64),
        "cdb_mw_l8_fp32_full": dict(full, solver="mwdg2", precision=32),
    }


def make_case(spec: dict, directory: str):
    """The benchmark's 4096^2 fBm catchment (the generator's defaults: 2 m cells, Hurst 0.8,
    relief 0-30 m, Manning 0.03, dry start, 50 m^3/s peak inflow at 30 min, epsilon 1e-3,
    seed 20261203), or the 256^2 circular dam break of the parity configuration (50 m
    square, flat bed, closed walls, 2.5 m inside radius 2.5 m, 0.5 m outside, epsilon 1e-3,
    3.5 s)."""
    if spec["kind"] == "catchment":
        return cases.fbm_catchment(directory, L=spec["L"], solver=spec["solver"])
    if spec["kind"] == "cdb":
        return cases.circular_dam_break(directory, L=spec["L"], solver=spec["solver"], sim_time=3.5, massint=None)
    raise ValueError(spec["kind"])


def run_case(name: str, spec: dict, ref_dir: str, out_dir: str) -> dict:
    work = tempfile.mkdtemp(prefix="digest_")
    try:
        c = make_case(spec, work)
        dig = os.path.join(work, "digest")
        os.makedirs(dig)
        exe = os.path.join(ref_dir, f"gpu-mwdg2-ref-fp{spec['precision']}")
        env = dict(os.environ, MWDG2_REF_DIGEST_DIR=dig,
                   MWDG2_REF_SAMPLE_STEPS=",".join(str(s) for s in spec["samples"]),
                   MWDG2_REF_STEPS_CSV=os.path.join(work, "steps.csv"))
        if spec["steps"] is not None:
            # the state after step n is sampled when step n + 1 starts
            env["MWDG2_REF_STOP_AFTER"] = str(spec["steps"] + 1)
        r = subprocess.run([exe, os.path.basename(c.par)], cwd=work, env=env, capture_output=True, text=True,
                           timeout=1800)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: reference exited {r.returncode}: {r.stderr[-2000:]}")
        rows = list(csv.DictReader(open(os.path.join(work, "steps.csv"))))
        nsteps = spec["steps"] if spec["steps"] is not None else len(rows)
        rows = rows[:nsteps]
        table = np.zeros((nsteps, len(NAMES)), np.uint64)
        present = np.zeros(len(NAMES), bool)
        for rw in csv.DictReader(open(os.path.join(dig, "digest.csv"))):
            s = int(rw["step"])
            if s > nsteps:
                continue
            k = NAMES.index(rw["name"])
            table[s - 1, k] = np.uint64(int(rw["hash"]))
            present[k] = True
        out = {"names": np.array(NAMES), "present": present, "digest": table,
               "steps_dt": np.array([float(rw["dt"]) for rw in rows]),
               "steps_n": np.array([int(rw["n_leaves"]) for rw in rows], np.int64)}
        real = np.float64 if spec["precision"] == 64 else np.float32
        kept = []
        for s in spec["samples"]:
            path = os.path.join(dig, f"sample_step{s:06d}.bin")
            if s > nsteps or not os.path.exists(path):
                continue
            raw = open(path, "rb").read()
            nreal = (len(raw) - 12 * 8) // np.dtype(real).itemsize
            vals = np.frombuffer(raw[:nreal * np.dtype(real).itemsize], real).reshape(12, -1)
            out[f"sample_{s}"] = vals
            out[f"sums_{s}"] = np.frombuffer(raw[nreal * np.dtype(real).itemsize:], np.float64)
            kept.append(s)
        out["sample_steps"] = np.array(kept, np.int32)
        dst = os.path.join(out_dir, f"digest_{name}.npz")
        np.savez_compressed(dst, **out)
        return {"name": name, "spec": spec, "steps": nsteps, "samples": kept, "bytes": os.path.getsize(dst)}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--ref-dir", default=os.path.join(ROOT, "oracle", "_ref"))
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    index_path = os.path.join(a.out, "digest_index.json")
    index = json.load(open(index_path)) if os.path.exists(index_path) else []
    for name, spec in case_specs().items():
        if a.only and a.only not in name:
            continue
        info = run_case(name, spec, a.ref_dir, a.out)
        print(json.dumps(info), flush=True)
        index = [e for e in index if e["name"] != name] + [info]
    with open(index_path, "w") as fp:
        json.dump(sorted(index, key=lambda e: e["name"]), fp, indent=1)


if __name__ == "__main__":
    main()
