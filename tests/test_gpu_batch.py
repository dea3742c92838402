"""Batched ensembles (mwdg2_batch_*): members stepped together equal the same cases run alone.

Every kernel of a step is deterministic (the wet-list order varies between runs, but each
leaf's update is independent of it and the dt and maxima reductions are exact), so a
member of a batch must reproduce a standalone run of its case bit for bit: the same dt
sequence, leaf grids and states. The members differ in size, solver, friction and limiter,
and one ends earlier than the others. From their second step on, members of one size class
(MWDG2, the same max_ref_lvl and precision, up to the batch's class level; none by default)
take one launch per kernel for the whole class (a member table, one member per blockIdx.y);
the others step on their own. The first test runs without and with classes (the two L = 7
MWDG2 members form one); the second holds a class of three max_ref_lvl 11 members (per-level
kernels above the bands, the value decode beside the leaf topology) to their standalone
runs."""
import os

import numpy as np
import pytest

import cases
import mwdg2_b200

pytestmark = pytest.mark.gpu


def _members(root: str):
    out = []
    d = os.path.join(root, "cdb7")
    out.append(cases.circular_dam_break(d, L=7, solver="mwdg2", sim_time=0.6, massint=None).par)
    d = os.path.join(root, "fbm7")
    z = cases.fbm_surface(128, 0.8, 7, 30.0)
    out.append(cases.fbm_catchment(d, L=7, solver="mwdg2", cellsize=2.0, sim_time=5.0, manning=0.03, peak_q=50.0,
                                   t_peak=300.0, start_depth=np.maximum(0.0, 12.0 - z), limitslopes=True).par)
    d = os.path.join(root, "cdb6hw")
    out.append(cases.circular_dam_break(d, L=6, solver="hwfv1", sim_time=0.2, massint=None).par)
    return out


@pytest.mark.parametrize("precision,group_level", [(64, 0), (32, 0), (64, 9), (32, 9)])
def test_batch_members_equal_standalone_runs(tmp_path, precision, group_level):
    pars = _members(str(tmp_path))
    steps = 25
    alone = []
    for p in pars:
        s = mwdg2_b200.Simulation(p, precision=precision)
        dts = []
        for _ in range(steps):
            ok, dt, n = s.step()
            if not ok:
                break
            dts.append(dt)
        alone.append((dts, s.leaves(), s.state()))
        s.close()
    with mwdg2_b200.Batch(pars, precision=precision) as b:
        b.group_max_level(group_level)
        dts = [[] for _ in pars]
        for _ in range(steps):
            k, dt, n = b.step()
            for i in range(len(pars)):
                if n[i]:
                    dts[i].append(dt[i])
        assert len(dts[2]) < steps, "the short member should have finished inside the window"
        for i, (want_dts, want_leaves, want_state) in enumerate(alone):
            m = b.member(i)
            assert dts[i] == want_dts, f"member {i}: dt sequence"
            got = m.leaves()
            for key in want_leaves:
                np.testing.assert_array_equal(got[key], want_leaves[key], err_msg=f"member {i}: {key}")
            st = m.state()
            for key in want_state:
                np.testing.assert_array_equal(st[key], want_state[key], err_msg=f"member {i}: {key}")
        # stepping on after every member is done reports DONE with no member stepped
        b.run()
        k, _, n = b.step()
        assert k == 0 and not n.any()


def _run_alone(pars, precision, steps):
    alone = []
    for p in pars:
        s = mwdg2_b200.Simulation(p, precision=precision)
        dts = []
        for _ in range(steps):
            ok, dt, n = s.step()
            if not ok:
                break
            dts.append(dt)
        alone.append((dts, s.leaves(), s.state()))
        s.close()
    return alone


@pytest.mark.parametrize("precision", [32, 64])
def test_size_class_members_equal_standalone_runs(tmp_path, precision):
    L = 11
    root = str(tmp_path)
    z = cases.fbm_surface(1 << L, 0.8, 11, 30.0)
    pars = [cases.fbm_catchment(os.path.join(root, "dry"), L=L, sim_time=600.0, peak_q=50.0, t_peak=30.0).par,
            cases.fbm_catchment(os.path.join(root, "wet"), L=L, sim_time=600.0, peak_q=0.0, manning=0.02,
                                start_depth=np.maximum(0.0, 9.00037 - z), limitslopes=True).par,
            cases.fbm_catchment(os.path.join(root, "short"), L=L, sim_time=0.5, peak_q=20.0, t_peak=30.0,
                                hurst=0.7, seed=5).par]
    steps = 8
    alone = _run_alone(pars, precision, steps)
    with mwdg2_b200.Batch(pars, precision=precision) as b:
        b.group_max_level(L)   # classes hold members up to 512^2 by default
        dts = [[] for _ in pars]
        for _ in range(steps):
            k, dt, n = b.step()
            for i in range(len(pars)):
                if n[i]:
                    dts[i].append(dt[i])
        for i, (want_dts, want_leaves, want_state) in enumerate(alone):
            m = b.member(i)
            assert dts[i] == want_dts, f"member {i}: dt sequence"
            got = m.leaves()
            for key in want_leaves:
                np.testing.assert_array_equal(got[key], want_leaves[key], err_msg=f"member {i}: {key}")
            st = m.state()
            for key in want_state:
                np.testing.assert_array_equal(st[key], want_state[key], err_msg=f"member {i}: {key}")
            assert m.last_step_counters()["launches"] > 0
