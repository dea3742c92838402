"""Monai valley functional test of the reference (cases/monai), through the drop-in entry.

The case runs the `monai` non-reflecting wave maker on the west boundary, `refine_wall`
preflags along the north and east walls, and Manning friction on a 392 x 243 laboratory
bathymetry at max_ref_lvl 9 for 22.5 s (about 6000 steps). The reference ships the stage
series an earlier build of it wrote for HWFV1 and MWDG2 at epsilon 0 and 1e-3 and judges
a build by the mean absolute depth error at the second gauge (run-functional-tests.py, no
threshold). Against those series every gauge is compared: the 226 output times within
0.01 s (dt differs in the last digits, so an output lands a step earlier or later), and
the mean absolute depth error at most 2.5e-4 m. The reference's own current build misses
its shipped series by as much (3e-5 to 1.8e-4 m; depths are 0.01-0.03 m), so when that
build is present (oracle/_ref) the same inputs also run through it live: then this build's
error may not exceed the live build's by more than 1e-5 m, and the two res.stage files
(6 printed decimals) must agree to within 1e-5 m on average and 2e-4 m at any sample.
At epsilon 0 they are identical; in the adaptive MWDG2 run, last-bit differences of fused
multiply-adds flip an occasional significance decision over the 6000 steps, and single
samples then differ by up to 9e-5 m while the means agree to 1e-6 m."""
import os
import subprocess

import numpy as np
import pytest

import make_golden_monai
import mwdg2_b200

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "gpu-mwdg2-ref-fp64")
MEAN_TOL = 2.5e-4
LIVE_TOL = 2e-4
LIVE_MEAN_TOL = 1e-5
LIVE_SLACK = 1e-5
TIME_TOL = 0.01


def _series(path: str) -> np.ndarray:
    return np.loadtxt(path, skiprows=9)


def _run_ours(d: str, par: str) -> np.ndarray:
    cwd = os.getcwd()
    os.chdir(d)
    try:
        st = mwdg2_b200.run_simulation(["gpu-mwdg2", "-precision", "64", os.path.basename(par)])
    finally:
        os.chdir(cwd)
    assert st == 0, mwdg2_b200.lib().mwdg2_last_error().decode()
    return _series(os.path.join(d, "res", "res.stage"))


@pytest.mark.parametrize("solver,eps", make_golden_monai.RUNS, ids=[f"{s}-eps-{e}" for s, e in make_golden_monai.RUNS])
def test_monai_stage_series_matches_reference(tmp_path, solver, eps):
    g = np.load(make_golden_monai.FIXTURE)
    par = make_golden_monai.write_case(str(tmp_path / "ours"), solver, eps, g)
    mine = _run_ours(str(tmp_path / "ours"), par)
    gold = make_golden_monai.golden_series(solver, eps, g)
    assert mine.shape == gold.shape
    stats = {"time_max_diff": float(np.abs(mine[:, 0] - gold[:, 0]).max()),
             "golden_mean_abs": np.abs(mine[:, 1:] - gold[:, 1:]).mean(axis=0).tolist()}
    if os.path.exists(REF):
        d = str(tmp_path / "ref")
        rpar = make_golden_monai.write_case(d, solver, eps, g)
        r = subprocess.run([REF, os.path.basename(rpar)], cwd=d, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        live = _series(os.path.join(d, "res", "res.stage"))
        assert live.shape == mine.shape
        stats["live_max_abs"] = float(np.abs(live - mine).max())
        stats["live_mean_abs"] = float(np.abs(live[:, 1:] - mine[:, 1:]).mean())
        stats["live_vs_golden_mean_abs"] = np.abs(live[:, 1:] - gold[:, 1:]).mean(axis=0).tolist()
    ok = stats["time_max_diff"] <= TIME_TOL and max(stats["golden_mean_abs"]) <= MEAN_TOL
    ok = ok and stats.get("live_max_abs", 0.0) <= LIVE_TOL and stats.get("live_mean_abs", 0.0) <= LIVE_MEAN_TOL
    if "live_vs_golden_mean_abs" in stats:
        ok = ok and all(m <= l + LIVE_SLACK for m, l in zip(stats["golden_mean_abs"], stats["live_vs_golden_mean_abs"]))
    assert ok, " ".join(f"{k}={v}" for k, v in stats.items())


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference build (oracle/_ref) is not present")
@pytest.mark.parametrize("solver", ["hwfv1", "mwdg2"])
def test_oregon_wave_maker_matches_reference_build(tmp_path, solver):
    """The oregon-seaside wave maker (west HFIX/HVAR ghost velocity 2 s(t) - v) has no
    shipped series: the Monai inputs with `oregon-seaside` in place of `monai`, 3 s at
    epsilon 0, run through this build and the reference build must give identical stage
    files (6 printed decimals)."""
    g = np.load(make_golden_monai.FIXTURE)
    out = {}
    for who in ("ours", "ref"):
        d = str(tmp_path / who)
        par = make_golden_monai.write_case(d, solver, "0", g)
        text = open(par).read().replace("monai\n", "oregon-seaside\n", 1).replace("sim_time      22.5", "sim_time      3.0")
        with open(par, "w") as fp:
            fp.write(text)
        if who == "ours":
            out[who] = _run_ours(d, par)
        else:
            r = subprocess.run([REF, os.path.basename(par)], cwd=d, capture_output=True, text=True, timeout=900)
            assert r.returncode == 0, r.stderr[-2000:]
            out[who] = _series(os.path.join(d, "res", "res.stage"))
    assert out["ours"].shape == out["ref"].shape
    assert np.abs(out["ours"] - out["ref"]).max() <= 1e-6
