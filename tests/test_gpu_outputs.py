"""saveint outputs (raster maps, VTK, c-prop CSVs, res.cumu) against the reference build.

The reference's own run_simulation wrote the golden files (tests/golden/out_*.npz, made
by make_golden_outputs.py); the product writes the same case through the drop-in entry
mwdg2_run_simulation. File names and every non-numeric line must match exactly; numbers
match within the state tolerances of the step parity tests, relative to max(1, |value|):
1e-9 (FP64) and 5e-5 (FP32), plus one unit of the last printed decimal (6 decimals in
VTK files and res.cumu: two values a hair apart can round to neighbouring decimals).
Velocity maps (.vx, .vy) divide by depths down to tol_h = 1e-3, which magnifies absolute
errors of the state by up to 1/tol_h, so their tolerance is 1e3 times larger. The runtime columns of res.cumu are host timings and are not
compared."""
import os
import re

import numpy as np
import pytest

import make_golden_outputs
import mwdg2_b200

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
TOL = {64: 1e-9, 32: 5e-5}
NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?|nan|inf", re.IGNORECASE)


def _split(text: str):
    """Lines of a text output: (template with numbers replaced, numbers)."""
    out = []
    for line in text.splitlines():
        nums = [float(x) for x in NUM.findall(line)]
        out.append((NUM.sub("#", line), nums))
    return out


def _decimals(name: str) -> float:
    return 1e-6 if name.endswith((".vtk", ".cumu")) else 0.0


def _compare(name: str, mine: str, ref: str, tol: float):
    a, b = _split(mine), _split(ref)
    assert len(a) == len(b), f"{name}: {len(a)} lines, reference {len(b)}"
    worst = 0.0
    for k, ((ta, na), (tb, nb)) in enumerate(zip(a, b)):
        assert ta == tb, f"{name} line {k + 1}: {ta[:80]!r} vs {tb[:80]!r}"
        if name.endswith(".cumu") and k > 0:
            na, nb = [na[0], na[4], na[5]], [nb[0], nb[4], nb[5]]   # simtime, dt, reduction
        x, y = np.array(na), np.array(nb)
        if x.size:
            err = np.abs(x - y) - _decimals(name)
            worst = max(worst, float(np.max(err / np.maximum(1.0, np.abs(y)))))
    assert worst <= tol, f"{name}: worst relative difference {worst:.3e} > {tol:.0e}"


@pytest.mark.parametrize("name", sorted(make_golden_outputs.output_specs()))
def test_saveint_outputs_match_reference(name, tmp_path):
    kind, solver, L, prec, kws = make_golden_outputs.output_specs()[name]
    gold = np.load(os.path.join(GOLDEN, name + ".npz"))
    ref = {k: bytes(gold[k]).decode() for k in gold.files}
    c = make_golden_outputs.make_output_case(str(tmp_path), kind, solver, L, kws)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        st = mwdg2_b200.run_simulation(["gpu-mwdg2", "-precision", str(prec), os.path.basename(c.par)])
    finally:
        os.chdir(cwd)
    assert st == 0, mwdg2_b200.lib().mwdg2_last_error().decode()
    mine = make_golden_outputs.collect_outputs(str(tmp_path))
    assert sorted(mine) == sorted(ref)
    for f in sorted(ref):
        _compare(f, mine[f], ref[f], TOL[prec] * (1e3 if f.endswith((".vx", ".vy")) else 1.0))
