"""The CPU oracle's keep-values decode (the checker of the library's mwdg2_set_decode_mode 1)
against its reference decode: the same trees step after step and states within 1e-10
relative in FP64 (the decodes differ by the round trip's rounding only), and in FP32 the
water of the FP64 run at the same simulated time, where the reference decode's round trip
of eta = h + z leaves depths of either sign in the dry cells."""
import numpy as np
import pytest

import cases
import oracle_py
from gpu_util import FIELDS, rel_err


@pytest.mark.parametrize("solver", ["mwdg2", "hwfv1"])
def test_oracle_keep_values_follows_reference_decode(tmp_path, solver):
    c = cases.fbm_catchment(str(tmp_path), L=7, solver=solver, sim_time=600.0, peak_q=50.0, t_peak=60.0,
                            limitslopes=(solver == "mwdg2"))
    ref, keep = oracle_py.Oracle(c.par, 64), oracle_py.Oracle(c.par, 64)
    keep.set_keep_values(True)
    for s in range(1, 31):
        assert ref.step()[0] and keep.step()[0]
        lr, lk = ref.leaves(), keep.leaves()
        for k in ("act", "lvl", "nb_ids", "nb_lvls"):
            np.testing.assert_array_equal(lk[k], lr[k], err_msg=f"step {s} {k}")
        np.testing.assert_array_equal(keep.sig(), ref.sig(), err_msg=f"step {s} sig")
        sr, sk = ref.state(), keep.state()
        for f in FIELDS:
            assert rel_err(sk[f], sr[f]) <= 1e-10, f"step {s} {f}"


def test_oracle_keep_values_fp32_water(tmp_path):
    c = cases.fbm_catchment(str(tmp_path), L=7, solver="mwdg2", sim_time=20.0, peak_q=20.0, t_peak=60.0,
                            limitslopes=True)
    vol = {}
    for name, precision, keep in (("fp64", 64, False), ("fp32", 32, False), ("fp32keep", 32, True)):
        o = oracle_py.Oracle(c.par, precision)
        o.set_keep_values(keep)
        while o.step()[0]:
            pass
        info, st, lv = o.info(), o.state(), o.leaves()
        assert abs(info["current_time"] - 20.0) < 1e-4
        area = info["dx"] ** 2 * np.ldexp(1.0, 2 * (info["L"] - lv["lvl"].astype(np.int64)))
        vol[name] = float(np.sum(st["h0"] * area))
    assert abs(vol["fp32keep"] - vol["fp64"]) <= 1e-3 * vol["fp64"], vol
    assert abs(vol["fp32keep"] - vol["fp64"]) < abs(vol["fp32"] - vol["fp64"]), vol
