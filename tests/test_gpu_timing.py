"""Device timing modes (mwdg2_set_timing): none, step (two events around each step's device
work, outside its captured graph) and phases (events between the phases, captured into the
step's graph). Timing never changes results: the same case run with each mode gives the
same state bit for bit."""
import numpy as np
import pytest

import cases
import mwdg2_b200
from gpu_util import FIELDS

pytestmark = pytest.mark.gpu
STEPS = 6


def _run(par: str, mode):
    sim = mwdg2_b200.Simulation(par, precision=32, timing=mode)
    times = []
    for _ in range(STEPS):
        assert sim.step()[0]
        times.append(sim.last_step_timing())
    st = sim.state()
    sim.close()
    return np.array(times), st


def test_timing_modes(tmp_path):
    c = cases.circular_dam_break(str(tmp_path), L=8)
    t_none, s_none = _run(c.par, False)
    t_step, s_step = _run(c.par, "step")
    t_ph, s_ph = _run(c.par, "phases")
    assert not t_none.any()
    # step mode: the whole step only; phases: every phase and the whole step
    assert (t_step[:, 7] > 0).all() and not t_step[:, :7].any()
    assert (t_ph[:, 7] > 0).all() and (t_ph[:, 1:7] > 0).all()
    # the phases lie inside the step
    assert (t_ph[:, :7].sum(axis=1) <= t_ph[:, 7] * 1.001 + 1e-3).all()
    for f in FIELDS:
        np.testing.assert_array_equal(s_step[f], s_none[f], err_msg=f)
        np.testing.assert_array_equal(s_ph[f], s_none[f], err_msg=f)
