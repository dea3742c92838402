"""Failure detection on the device, driven by a corrupted host input (no GPU fault).

A start raster with one depth written as "nan" puts a NaN into the initial state. The
solver kernels flag NaN depths in the state they write (Scalars::status), the step's one
read-back carries the flag, and mwdg2_step returns MWDG2_ERR_NUMERIC instead of advancing
with a corrupted state; the handle stays usable for the getters and mwdg2_destroy."""
import pytest

import cases
import mwdg2_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
def test_nan_in_start_raster_gives_numeric_error(tmp_path, solver):
    c = cases.start_q_nodata(str(tmp_path), L=7, solver=solver, nan_cell=True)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    try:
        with pytest.raises(mwdg2_b200.MWDG2Error) as err:
            for _ in range(5):
                sim.step()
        assert err.value.status == 4, str(err.value)
        assert sim.info()["L"] == 7
    finally:
        sim.close()


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
def test_same_case_without_nan_steps(tmp_path, solver):
    c = cases.start_q_nodata(str(tmp_path), L=7, solver=solver, nan_cell=False)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    try:
        for _ in range(5):
            ok, dt, n = sim.step()
            assert ok and dt > 0 and n > 0
    finally:
        sim.close()
