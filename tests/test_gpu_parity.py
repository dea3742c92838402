"""CUDA path against the reference's own CUDA build (golden fixtures) and the CPU oracle.

Bit-exact: leaf lists, levels, neighbour ids and levels, significance flags (every
dumped step). State errors are measured relative to max(1, |value|):
  * FP64: 1e-10 against the reference build and against the oracle, every step;
  * FP32 against the FP32 reference build over 40 steps: 2e-5; against the FP32 oracle
    (no fused multiply-adds) over 15 steps: 1e-4 -- single-precision rounding differences
    between two IEEE evaluations grow through the moving shock;
  * FP32 against the FP64 oracle after one step from the same inputs: 1e-5, with depth
    errors scaled by the free-surface elevation |h| + |z| the state stores (h = eta - z
    loses the low bits of eta by cancellation over high ground).
dt within 1e-9 (FP64) / 2e-5 (FP32). Calls go through the C ABI (include/mwdg2.h)."""
import os
import re
import tempfile

import numpy as np
import pytest

import make_golden
import mwdg2_b200
import oracle_py
from gpu_util import FIELDS, assert_same_topology, rel_err

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
TOL = {64: 1e-10, 32: 2e-5}
TOL_ORACLE = {64: 1e-10, 32: 1e-4}
DT_TOL = {64: 1e-9, 32: 2e-5}


def _cases():
    return sorted(make_golden.case_specs().items())


def _golden_topology(g, s):
    out = {"act": g[f"s{s}_leaf_act"], "lvl": g[f"s{s}_leaf_lvl"],
           "nb_ids": np.stack([g[f"s{s}_nb_{d}_ids"] for d in "nesw"])}
    if f"s{s}_nb_n_lvls" in g:
        out["nb_lvls"] = np.stack([g[f"s{s}_nb_{d}_lvls"] for d in "nesw"])
    return out


@pytest.mark.parametrize("name,spec", _cases(), ids=[n for n, _ in _cases()])
def test_cuda_matches_reference_build(name, spec):
    kw, prec = spec
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    last = max(int(k.split("_")[0][1:]) for k in g.files if re.match(r"^s\d+_", k))
    with tempfile.TemporaryDirectory() as d:
        c = make_golden.make_case(kw["kind"], d, kw["L"], kw["solver"])
        sim = mwdg2_b200.Simulation(c.par, precision=prec)
        dts, ns = [], []
        for s in range(1, last + 1):
            ok, dt, n = sim.step()
            assert ok
            dts.append(dt)
            ns.append(n)
            if f"s{s}_leaf_act" not in g:
                continue
            lv = sim.leaves()
            ref = _golden_topology(g, s)
            if "nb_lvls" not in ref:
                lv.pop("nb_lvls")
            assert_same_topology(lv, ref, f"{name} step {s}")
            np.testing.assert_array_equal(sim.sig(), g[f"s{s}_sig"], err_msg=f"{name} step {s} sig")
            if f"s{s}_state_h0" in g:
                st = sim.state()
                idx = g[f"s{s}_state_idx"] if f"s{s}_state_idx" in g else slice(None)
                for f in FIELDS:
                    key = f"s{s}_state_{f}"
                    if key in g:
                        e = rel_err(st[f][idx], g[key])
                        assert e <= TOL[prec], f"{name} step {s} {f}: {e:.3e}"
        np.testing.assert_array_equal(np.array(ns), g["steps_n"][:last])
        assert rel_err(dts, g["steps_dt"][:last]) <= DT_TOL[prec]


@pytest.mark.parametrize("name,spec", _cases(), ids=[n for n, _ in _cases()])
def test_cuda_matches_oracle_every_step(name, spec):
    kw, prec = spec
    with tempfile.TemporaryDirectory() as d:
        c = make_golden.make_case(kw["kind"], d, kw["L"], kw["solver"])
        sim = mwdg2_b200.Simulation(c.par, precision=prec)
        orc = oracle_py.Oracle(c.par, prec)
        for s in range(1, 16):
            ok, dt, n = sim.step()
            ok2, dt2, n2 = orc.step()
            assert ok and ok2 and n == n2, f"{name} step {s}: leaves {n} vs {n2}"
            lv, lo = sim.leaves(), orc.leaves()
            if kw["solver"] == "hwfv1":
                lv.pop("nb_lvls"); lo.pop("nb_lvls")
            assert_same_topology(lv, lo, f"{name} step {s}")
            np.testing.assert_array_equal(sim.sig(), orc.sig())
            st, so = sim.state(), orc.state()
            for f in FIELDS:
                assert rel_err(st[f], so[f]) <= TOL_ORACLE[prec], f"{name} step {s} {f}"
            assert abs(dt - dt2) <= DT_TOL[prec] * dt2


@pytest.mark.parametrize("kind,solver", [("cdb", "mwdg2"), ("fbm", "mwdg2"), ("cdb", "hwfv1")])
def test_fp32_against_fp64_oracle_one_step(kind, solver):
    """FP32 state after one step within 1e-5 of the FP64 oracle on every leaf both grids share."""
    with tempfile.TemporaryDirectory() as d:
        c = make_golden.make_case(kind, d, 7, solver)
        sim = mwdg2_b200.Simulation(c.par, precision=32)
        orc = oracle_py.Oracle(c.par, 64)
        sim.step()
        orc.step()
        a, b = sim.leaves()["act"], orc.leaves()["act"]
        common, ia, ib = np.intersect1d(a, b, return_indices=True)
        assert len(common) >= 0.99 * len(b)
        st, so = sim.state(), orc.state()
        for f in FIELDS:
            a_, b_ = st[f][ia], so[f][ib]
            scale = np.maximum(1.0, np.abs(b_))
            if f.startswith("h"):
                zf = "z" + f[1:]
                scale = np.maximum(1.0, np.abs(b_) + np.abs(so[zf][ib]))
            e = float(np.max(np.abs(a_ - b_) / scale)) if a_.size else 0.0
            assert e <= 1e-5, f"{kind} {solver} {f}: {e:.3e}"


# Fraction of the step-1 leaf state (12 coefficients per leaf) that must be bit-identical
# to the reference build. Every formula keeps the reference's operand order, so nvcc forms
# the same fused multiply-adds wherever both builds see the same expression; the rest
# differ in the last bit. Observed: MWDG2 99.4-99.99 %, HWFV1 93.6-99.5 %; the case with an
# initial discharge (startq2d), where every leaf is wet and moving from the first step,
# 98.4 % (MWDG2) and 88.7 % (HWFV1).
BITS_MIN = {"mwdg2": 0.99, "hwfv1": 0.92}
BITS_MIN_CASE = {"startq_mw_l7_fp64": 0.98, "startq_hw_l7_fp64": 0.88}


@pytest.mark.parametrize("name,spec", _cases(), ids=[n for n, _ in _cases()])
def test_first_step_state_bit_identical_to_reference_build(name, spec):
    kw, prec = spec
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    word = np.uint32 if prec == 32 else np.uint64
    with tempfile.TemporaryDirectory() as d:
        c = make_golden.make_case(kw["kind"], d, kw["L"], kw["solver"])
        sim = mwdg2_b200.Simulation(c.par, precision=prec)
        assert sim.step()[0]
        st = sim.state()
    idx = g["s1_state_idx"] if "s1_state_idx" in g else slice(None)
    same = total = 0
    for f in FIELDS:
        key = f"s1_state_{f}"
        if key not in g:
            continue
        ftype = np.float32 if prec == 32 else np.float64
        a = np.ascontiguousarray(np.asarray(st[f][idx], dtype=np.float64).astype(ftype))
        b = np.ascontiguousarray(np.asarray(g[key], dtype=np.float64).astype(ftype))
        same += int((a.view(word) == b.view(word)).sum())
        total += a.size
    assert total > 0
    assert same >= BITS_MIN_CASE.get(name, BITS_MIN[kw["solver"]]) * total, f"{name}: {same}/{total} values bit-identical"
