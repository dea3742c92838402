"""Golden fixture of the reference's Monai valley functional test (cases/monai).

The reference ships, for its Monai valley case, the nodal bathymetry (bed-data.txt), the
boundary, series and stage-point files (monai.bci, monai.bdy, monai.stage) and the stage
series its own build produced for HWFV1 and MWDG2 at epsilon 0 and 1e-3
({solver}-eps-{eps}/res.txt), which its cases/monai/run-functional-tests.py compares by
mean absolute error. This script packs those files (as read from the reference, nothing
re-typed) into tests/golden/monai.npz:

    python tests/golden/make_golden_monai.py [--ref-cases <folder of the reference's cases>]

and `write_case` rebuilds the case inputs from the fixture: the DEM and start rasters as
cases/monai/raster.py derives them from the nodal bathymetry (datum shift, initial depth
to the 0.13535 m still-water level, NODATA nodes to 100 m, 4-node average per cell,
"%.15f" ESRI text), and the .par as run-functional-tests.py writes it.
"""
from __future__ import annotations

import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "monai.npz")
RUNS = (("hwfv1", "0"), ("hwfv1", "0.001"), ("mwdg2", "0"), ("mwdg2", "0.001"))


def pack(ref_cases: str, out: str = FIXTURE) -> None:
    d = os.path.join(ref_cases, "monai")
    bed = np.loadtxt(os.path.join(d, "bed-data.txt"), skiprows=1, usecols=2)
    arrays = {"bed_nodal": bed}
    for name in ("monai.bci", "monai.bdy", "monai.stage"):
        with open(os.path.join(d, name), "rb") as fp:
            arrays[name] = np.frombuffer(fp.read(), dtype=np.uint8)
    for solver, eps in RUNS:
        with open(os.path.join(d, f"{solver}-eps-{eps}", "res.txt"), "rb") as fp:
            arrays[f"golden_{solver}_{eps}"] = np.frombuffer(fp.read(), dtype=np.uint8)
    np.savez_compressed(out, **arrays)
    print(out, os.path.getsize(out), "bytes")


def _raster_text(nodal: np.ndarray) -> bytes:
    nrows, ncols = nodal.shape
    raster = 0.25 * (((nodal[:-1, :-1] + nodal[:-1, 1:]) + nodal[1:, :-1]) + nodal[1:, 1:])
    header = ("ncols        %s\nnrows        %s\nxllcorner    %s\nyllcorner    %s\ncellsize     %s\n"
              "NODATA_value -9999" % (ncols - 1, nrows - 1, 0, 0, 0.014))
    rows = [" ".join("%.15f" % v for v in row) for row in np.flipud(raster)]
    return (header + "\n" + "\n".join(rows) + "\n").encode()


def write_case(directory: str, solver: str, eps: str, fixture=None) -> str:
    """Write the Monai case for `solver` and epsilon text `eps`; returns the .par path."""
    g = fixture if fixture is not None else np.load(FIXTURE)
    os.makedirs(directory, exist_ok=True)
    bed = g["bed_nodal"].reshape(393, 244).T.copy()   # 244 node rows x 393 node columns
    bed *= -1
    bed += 0.13535
    start = np.maximum(0.13535 - bed, 0)
    bed[(bed - -30) < 1e-10] = 100
    with open(os.path.join(directory, "monai.dem"), "wb") as fp:
        fp.write(_raster_text(bed))
    with open(os.path.join(directory, "monai.start"), "wb") as fp:
        fp.write(_raster_text(start))
    for name in ("monai.bci", "monai.bdy", "monai.stage"):
        with open(os.path.join(directory, name), "wb") as fp:
            fp.write(bytes(g[name]))
    par = os.path.join(directory, "functional-test.par")
    with open(par, "w") as fp:
        fp.write("monai\n" + f"{solver}\n" + "cuda\n" + "cumulative\n" + "refine_wall\n" + "ref_thickness 16\n" +
                 "max_ref_lvl   9\n" + f"epsilon       {eps}\n" + "wall_height   0.5\n" + "initial_tstep 1\n" +
                 "fpfric        0.01\n" + "sim_time      22.5\n" + "massint       0.1\n" + "saveint       22.5\n" +
                 "DEMfile       monai.dem\n" + "startfile     monai.start\n" + "bcifile       monai.bci\n" +
                 "bdyfile       monai.bdy\n" + "stagefile     monai.stage\n")
    return par


def golden_series(solver: str, eps: str, fixture=None) -> np.ndarray:
    """Rows of (time, depth at stage 1, 2, 3) the reference's build wrote for this run."""
    g = fixture if fixture is not None else np.load(FIXTURE)
    text = bytes(g[f"golden_{solver}_{eps}"]).decode()
    return np.loadtxt(text.splitlines(), skiprows=9)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-cases", default=os.path.join(os.environ.get("MWDG2_REFERENCE", "/root/reference"), "cases"))
    pack(ap.parse_args().ref_cases)


if __name__ == "__main__":
    main()
