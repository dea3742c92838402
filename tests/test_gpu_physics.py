"""Physical invariants of the CUDA path as the reference's scheme has them, and parity on an
urban catchment (building blocks 5-20 m tall: wet/dry fronts against walls, fast flows).

* Well-balancing: a lake at rest over an fBm bed (fully wet) stays at rest. After 20 steps
  every leaf's discharge |q0| is at most 1e-12 (FP64) or 1e-5 (FP32), and its free surface
  h0 + z0 lies within 1e-12 (FP64) or 1e-4 (FP32, ~840 units in the last place of the 1 m
  level: fused multiply-adds make the per-step cancellation inexact) of the level.
* Mass: with epsilon 0 (every detail kept) and no limiter, the volume sum(h0 * cell area) of
  a closed dam break changes by at most 1e-13 (FP64) or 1e-7 (FP32) relative over 30 steps.
  With epsilon > 0 the volume drifts in the reference's scheme (its fluxes at resolution
  interfaces use the coarser side's ancestor values), so no bound is asserted there.
* Urban catchment against the CPU oracle (FP64, 10 steps): leaves, neighbours and
  significance flags bit-exact every step, state within 1e-10 relative to max(1, |value|),
  dt within 1e-9. The lake stands at 1.00037 m with depths written to 6 decimals: on the
  0.001 m lattice of a 3-decimal DEM, thin-water face depths land exactly on the 1e-3 dry
  threshold, where the wet/dry branch follows the last bit of the face value and hence
  the choice of fused multiply-adds (two IEEE CPU builds, with and without contraction,
  then differ by 1e-7 after one step); off the lattice the two agree to 2e-11 over 12 steps.
* Partly wet fBm catchment with Manning friction and the slope limiter against the CPU
  oracle (FP64, 12 steps, same bounds): valleys filled to a level off the DEM's 0.001 m
  lattice leave about 30 % of the leaves wet, so from step 2 both RK stages run the wet
  test, the dry-leaf writer and the wet-list kernel with friction on the listed leaves and
  their neighbours' copies.
Calls go through the C ABI (include/mwdg2.h)."""
import numpy as np
import pytest

import cases
import mwdg2_b200
import oracle_py
from gpu_util import FIELDS, assert_same_topology, rel_err

pytestmark = pytest.mark.gpu
Q_REST_TOL = {64: 1e-12, 32: 1e-5}
ETA_REST_TOL = {64: 1e-12, 32: 1e-4}
MASS_TOL = {64: 1e-13, 32: 1e-7}


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
@pytest.mark.parametrize("precision", [64, 32])
def test_lake_at_rest_stays_at_rest(tmp_path, solver, precision):
    c = cases.lake_at_rest(str(tmp_path), L=8, solver=solver, sim_time=100.0, level=1.0)
    with mwdg2_b200.Simulation(c.par, precision=precision) as sim:
        for _ in range(20):
            ok, dt, n = sim.step()
            assert ok and dt > 0
        st = sim.state()
    q = max(np.abs(st["qx0"]).max(), np.abs(st["qy0"]).max())
    eta = np.abs(st["h0"] + st["z0"] - 1.0).max()
    assert (st["h0"] > 0).all()
    assert q <= Q_REST_TOL[precision], f"|q| {q:.3e}"
    assert eta <= ETA_REST_TOL[precision], f"|eta - 1| {eta:.3e}"


def _volume(sim, L, dx):
    st, lv = sim.state(), sim.leaves()
    area = (dx * np.exp2(L - lv["lvl"].astype(np.float64))) ** 2
    return float(np.sum(st["h0"] * area))


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
@pytest.mark.parametrize("precision", [64, 32])
def test_volume_conserved_without_thresholding(tmp_path, solver, precision):
    c = cases.circular_dam_break(str(tmp_path), L=7, solver=solver, eps=0.0, limitslopes=False,
                                 massint=None)
    with mwdg2_b200.Simulation(c.par, precision=precision) as sim:
        assert sim.step()[0]
        v0 = _volume(sim, c.L, c.cellsize)
        drift = 0.0
        for _ in range(30):
            assert sim.step()[0]
            drift = max(drift, abs(_volume(sim, c.L, c.cellsize) - v0) / v0)
    assert drift <= MASS_TOL[precision], f"relative volume change {drift:.3e}"


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
def test_urban_catchment_matches_oracle(tmp_path, solver):
    c = cases.urban_catchment(str(tmp_path), L=8, solver=solver, sim_time=100.0, lake_level=1.00037)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    orc = oracle_py.Oracle(c.par, 64)
    try:
        for s in range(1, 11):
            ok, dt, n = sim.step()
            ok2, dt2, n2 = orc.step()
            assert ok and ok2 and n == n2, f"step {s}: leaves {n} vs {n2}"
            lv, lo = sim.leaves(), orc.leaves()
            if solver == "hwfv1":
                lv.pop("nb_lvls")
                lo.pop("nb_lvls")
            assert_same_topology(lv, lo, f"urban {solver} step {s}")
            np.testing.assert_array_equal(sim.sig(), orc.sig(), err_msg=f"step {s} sig")
            st, so = sim.state(), orc.state()
            for f in FIELDS:
                e = rel_err(st[f], so[f])
                assert e <= 1e-10, f"step {s} {f}: {e:.3e}"
            assert abs(dt - dt2) <= 1e-9 * dt2
    finally:
        sim.close()
        orc.close()


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
@pytest.mark.parametrize("precision", [64, 32])
def test_device_volume_reduction_matches_host_sum(tmp_path, solver, precision):
    """mwdg2_volume (FP64 reduction on the device) equals the host's FP64 sum of h0 x leaf
    area over the leaf state, on an adaptive fBm catchment after a few steps."""
    c = cases.fbm_catchment(str(tmp_path), L=8, solver=solver, sim_time=600.0,
                            start_depth=np.maximum(0.0, 12.0 - cases.fbm_surface(256, 0.8, 5, 30.0)))
    with mwdg2_b200.Simulation(c.par, precision=precision) as sim:
        for _ in range(5):
            assert sim.step()[0]
        host = _volume(sim, c.L, c.cellsize)
        dev = sim.volume()
    assert host > 0
    assert abs(dev - host) <= 1e-12 * host, (dev, host)


def test_partly_wet_catchment_with_friction_matches_oracle(tmp_path):
    L = 9
    z = cases.fbm_surface(1 << L, 0.8, 20261203, 30.0)
    h0 = np.maximum(0.0, 12.00037 - z)
    c = cases.fbm_catchment(str(tmp_path), L=L, start_depth=h0, sim_time=600.0, manning=0.03, limitslopes=True)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    orc = oracle_py.Oracle(c.par, 64)
    listed = 0
    try:
        for s in range(1, 13):
            ok, dt, n = sim.step()
            ok2, dt2, n2 = orc.step()
            assert ok and ok2 and n == n2, f"step {s}: leaves {n} vs {n2}"
            wet = sim.last_step_counters()["wet_stage1"]
            listed += int(s > 1 and 0 < 2 * wet < n)
            assert_same_topology(sim.leaves(), orc.leaves(), f"catchment step {s}")
            np.testing.assert_array_equal(sim.sig(), orc.sig(), err_msg=f"step {s} sig")
            st, so = sim.state(), orc.state()
            for f in FIELDS:
                e = rel_err(st[f], so[f])
                assert e <= 1e-10, f"step {s} {f}: {e:.3e}"
            assert abs(dt - dt2) <= 1e-9 * dt2
    finally:
        sim.close()
        orc.close()
    assert listed == 11, f"stage 1 ran over the wet list in {listed} of steps 2-12"
