"""The CPU oracle against the reference's own CUDA build (golden fixtures).

Fixtures in tests/golden/ were produced by tests/golden/make_golden.py, which runs the
reference (al0vya/gpu-mwdg2 built for sm_100a under oracle/_ref) on seeded inputs and
records its leaf lists, neighbours, significance flags, dt and leaf state.
Tree and topology must match bit for bit; state within 1e-10 (FP64) or 2e-5 (FP32)
relative to max(1, |value|) -- the oracle evaluates the same formulas without fused
multiply-adds, the reference's CUDA build fuses them.
"""
import os
import re
import tempfile

import numpy as np
import pytest

import make_golden
import oracle_py

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
TOL = {64: 1e-10, 32: 2e-5}
DT_TOL = {64: 1e-9, 32: 2e-5}
FIELDS = ("h0", "qx0", "qy0", "z0", "h1x", "qx1x", "qy1x", "z1x", "h1y", "qx1y", "qy1y", "z1y")


def _cases():
    return sorted(make_golden.case_specs().items())


@pytest.mark.parametrize("name,spec", _cases(), ids=[n for n, _ in _cases()])
def test_oracle_matches_reference(name, spec):
    kw, prec = spec
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    g = np.load(path)
    with tempfile.TemporaryDirectory() as d:
        c = make_golden.make_case(kw["kind"], d, kw["L"], kw["solver"])
        o = oracle_py.Oracle(c.par, prec)
        dts, ns = [], []
        last = max(int(k.split("_")[0][1:]) for k in g.files if re.match(r"^s\d+_", k))
        for s in range(1, last + 1):
            ok, dt, n = o.step()
            assert ok
            dts.append(dt)
            ns.append(n)
            if f"s{s}_leaf_act" not in g:
                continue
            lv = o.leaves()
            np.testing.assert_array_equal(lv["act"], g[f"s{s}_leaf_act"], err_msg=f"{name} step {s} act")
            np.testing.assert_array_equal(lv["lvl"], g[f"s{s}_leaf_lvl"], err_msg=f"{name} step {s} lvl")
            for i, dname in enumerate("nesw"):
                np.testing.assert_array_equal(lv["nb_ids"][i], g[f"s{s}_nb_{dname}_ids"])
                if f"s{s}_nb_{dname}_lvls" in g:
                    np.testing.assert_array_equal(lv["nb_lvls"][i], g[f"s{s}_nb_{dname}_lvls"])
            np.testing.assert_array_equal(o.sig(), g[f"s{s}_sig"], err_msg=f"{name} step {s} sig")
            if f"s{s}_state_h0" in g:
                st = o.state()
                idx = g[f"s{s}_state_idx"] if f"s{s}_state_idx" in g else slice(None)
                for f in FIELDS:
                    key = f"s{s}_state_{f}"
                    if key not in g:
                        continue
                    ref = g[key].astype(np.float64)
                    mine = st[f][idx]
                    err = np.abs(mine - ref) / np.maximum(1.0, np.abs(ref))
                    assert err.max() <= TOL[prec], f"{name} step {s} {f}: {err.max():.3e}"
                    tot = st[f].sum()
                    rsum = float(g[key + "_sum"][0])
                    assert abs(tot - rsum) <= TOL[prec] * max(1.0, np.abs(st[f]).sum()), f"{name} {f} sum"
        np.testing.assert_array_equal(np.array(ns), g["steps_n"][:last])
        rel = np.abs(np.array(dts) - g["steps_dt"][:last]) / g["steps_dt"][:last]
        assert rel.max() <= DT_TOL[prec]
