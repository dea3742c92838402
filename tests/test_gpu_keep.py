"""The keep-values decode (mwdg2_set_decode_mode 1): the children of a parent that the step's
encode visited keep the values the encode read, and only the parents refined this step are
decoded (no counterpart in the reference, whose decode returns those children only up to
rounding, mra/decoding.cu:3-67).

* Against the CPU oracle's keep-values option (FP64): leaves, neighbours and significance
  flags bit-exact every step, state within 1e-10 relative to max(1, |value|), dt within
  1e-9, on a partly wet fBm catchment with Manning friction and the slope limiter (wet-list
  stages from step 2) and on a dry-start catchment with a point inflow, MWDG2 and HWFV1;
  the MWDG2 runs leave the leaves that stay dry as they stand (frozen: the oracle writes
  them, to the same values up to the last bit of eta = h + z), and their scale re-encode
  keeps the parents whose children all stand (the oracle computes them again).
* Against this library's reference decode (FP64, 30 steps of the inflow catchment): the
  same trees every step and states within 1e-9 relative: the two decodes differ by the
  round trip's rounding only.
* A lake at rest over an fBm bed stays at rest (the bounds of the reference decode).
* With the learned refinement proposal: a proposal that keeps every subtree (the masked
  encode, decode and re-encode kernels with an all-ones mask) gives the keep-values step's
  results bit for bit.
* FP32 water: on the inflow catchment at t = 20 s (~200 steps) the FP32 run with the
  keep-values decode holds the FP64 run's water volume within 0.1 % (the CPU oracle: 5e-5),
  closer than the FP32 run with the reference decode, whose round trip of eta = h + z over
  the rough bed leaves depths of either sign in the dry cells every step (the oracle: 17 m^3
  of |depth| below 1 mm against 0.03 m^3 with the keep-values decode and in FP64).
Calls go through the C ABI (include/mwdg2.h)."""
import numpy as np
import pytest

import cases
import mwdg2_b200
import oracle_py
from gpu_util import FIELDS, assert_same_topology, rel_err

pytestmark = pytest.mark.gpu


def _partly_wet(tmp_path, solver):
    L = 9 if solver == "mwdg2" else 8
    z = cases.fbm_surface(1 << L, 0.8, 20261203, 30.0)
    return cases.fbm_catchment(str(tmp_path), L=L, solver=solver, start_depth=np.maximum(0.0, 12.00037 - z),
                               sim_time=600.0, manning=0.03, limitslopes=(solver == "mwdg2"))


def _inflow(tmp_path, solver):
    return cases.fbm_catchment(str(tmp_path), L=8, solver=solver, sim_time=600.0, peak_q=50.0, t_peak=60.0,
                               limitslopes=(solver == "mwdg2"))


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
@pytest.mark.parametrize("case", ["partly_wet", "inflow"])
def test_keep_values_matches_oracle(tmp_path, solver, case):
    c = (_partly_wet if case == "partly_wet" else _inflow)(tmp_path, solver)
    steps = 12 if case == "partly_wet" else 40
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    orc = oracle_py.Oracle(c.par, 64)
    sim.set_decode_mode("keep")
    orc.set_keep_values(True)
    frozen = 0
    try:
        for s in range(1, steps + 1):
            ok, dt, n = sim.step()
            ok2, dt2, n2 = orc.step()
            assert ok and ok2 and n == n2, f"step {s}: leaves {n} vs {n2}"
            frozen += sim.last_step_counters()["frozen_leaves"]
            lv, lo = sim.leaves(), orc.leaves()
            if solver == "hwfv1":
                lv.pop("nb_lvls")
                lo.pop("nb_lvls")
            assert_same_topology(lv, lo, f"{case} {solver} step {s}")
            np.testing.assert_array_equal(sim.sig(), orc.sig(), err_msg=f"step {s} sig")
            st, so = sim.state(), orc.state()
            for f in FIELDS:
                e = rel_err(st[f], so[f])
                assert e <= 1e-10, f"step {s} {f}: {e:.3e}"
            assert abs(dt - dt2) <= 1e-9 * dt2
    finally:
        sim.close()
        orc.close()
    # MWDG2 steps with both stages over the wet list freeze the leaves that stay dry
    assert (frozen > 0) == (solver == "mwdg2"), frozen


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
def test_keep_values_follows_reference_decode(tmp_path, solver):
    c = _inflow(tmp_path, solver)
    ref = mwdg2_b200.Simulation(c.par, precision=64)
    keep = mwdg2_b200.Simulation(c.par, precision=64)
    keep.set_decode_mode("keep")
    try:
        for s in range(1, 31):
            ok, dt, n = ref.step()
            ok2, dt2, n2 = keep.step()
            assert ok and ok2 and n == n2, f"step {s}: leaves {n} vs {n2}"
            lk, lr = keep.leaves(), ref.leaves()
            if solver == "hwfv1":
                lk.pop("nb_lvls")
                lr.pop("nb_lvls")
            assert_same_topology(lk, lr, f"keep vs reference decode, step {s}")
            st, sr = keep.state(), ref.state()
            for f in FIELDS:
                e = rel_err(st[f], sr[f])
                assert e <= 1e-9, f"step {s} {f}: {e:.3e}"
    finally:
        ref.close()
        keep.close()


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
@pytest.mark.parametrize("precision", [64, 32])
def test_keep_values_lake_at_rest(tmp_path, solver, precision):
    c = cases.lake_at_rest(str(tmp_path), L=8, solver=solver, sim_time=100.0, level=1.0)
    with mwdg2_b200.Simulation(c.par, precision=precision) as sim:
        sim.set_decode_mode("keep")
        for _ in range(20):
            ok, dt, n = sim.step()
            assert ok and dt > 0
        st = sim.state()
    q = max(np.abs(st["qx0"]).max(), np.abs(st["qy0"]).max())
    eta = np.abs(st["h0"] + st["z0"] - 1.0).max()
    assert (st["h0"] > 0).all()
    assert q <= {64: 1e-12, 32: 1e-5}[precision], f"|q| {q:.3e}"
    assert eta <= {64: 1e-12, 32: 1e-4}[precision], f"|eta - 1| {eta:.3e}"


def _constant_mlp(logit: float) -> np.ndarray:
    p = np.zeros(mwdg2_b200.MLP_PARAMS, np.float32)
    p[-4:] = logit
    return p


def test_keep_values_with_all_ones_proposal(tmp_path):
    c = _partly_wet(tmp_path, "mwdg2")
    runs = []
    for learned in (False, True):
        sim = mwdg2_b200.Simulation(c.par, precision=64)
        sim.set_decode_mode("keep")
        if learned:
            sim.proposal_record(True)
            sim.proposal_enable(_constant_mlp(20.0), judge_every=0, threshold=0.0, miss_bound=1.0)
        out = []
        for _ in range(6):
            assert sim.step()[0]
            out.append((sim.leaves(), sim.sig(), sim.state()))
        if learned:
            st = sim.proposal_stats()
            assert st["applied"] == 1.0 and st["proposed"] == st["subtrees"]
        sim.close()
        runs.append(out)
    for s, (x, y) in enumerate(zip(*runs)):
        assert_same_topology(y[0], x[0], f"all-ones proposal with keep values, step {s + 1}")
        np.testing.assert_array_equal(y[1], x[1], err_msg=f"step {s + 1}: flags")
        for f in FIELDS:
            np.testing.assert_array_equal(y[2][f], x[2][f], err_msg=f"step {s + 1}: {f}")


def _volumes(sim):
    """Water volume of the leaves (m^3) and the part of it in leaves less than 1 mm deep
    (absolute depths: the dry cells' depths of either sign)."""
    info = sim.info()
    st, lv = sim.state(), sim.leaves()
    area = info["dx"] ** 2 * np.ldexp(1.0, 2 * (info["L"] - lv["lvl"].astype(np.int64)))
    h = st["h0"]
    return float(np.sum(h * area)), float(np.sum(np.where(np.abs(h) < 1e-3, np.abs(h), 0.0) * area))


def test_keep_values_fp32_holds_the_fp64_water(tmp_path):
    # every run ends exactly at t = 20 s (the last step lands on sim_time), ~200 steps
    c = cases.fbm_catchment(str(tmp_path), L=8, solver="mwdg2", sim_time=20.0, peak_q=50.0, t_peak=60.0,
                            limitslopes=True)
    vol, thin = {}, {}
    for name, precision, mode in (("fp64", 64, "reference"), ("fp32", 32, "reference"), ("fp32keep", 32, "keep")):
        with mwdg2_b200.Simulation(c.par, precision=precision) as sim:
            sim.set_decode_mode(mode)
            while sim.step()[0]:
                pass
            assert abs(sim.info()["time"] - 20.0) < 1e-4
            vol[name], thin[name] = _volumes(sim)
    assert vol["fp64"] > 0
    err_keep = abs(vol["fp32keep"] - vol["fp64"])
    err_ref = abs(vol["fp32"] - vol["fp64"])
    assert err_keep <= 1e-3 * vol["fp64"], (vol, thin)
    assert err_keep < err_ref, (vol, thin)
    # the reference decode's round trip leaves depths in the dry cells; the keep-values decode
    # leaves the thin water of the FP64 run
    assert thin["fp32keep"] <= 0.1 * thin["fp32"], (vol, thin)
