"""The learned refinement proposal inside the time step (MWDG2, max_ref_lvl 11 fBm
catchment, FP64), through the C ABI:

* recording the features and activity labels leaves every result bit-identical;
* a proposal that keeps every subtree gives the plain step's results bit for bit (the masked
  encode, decode and re-encode kernels with an all-ones mask; the MLP run on every coarse
  cell, as with recording on);
* an MLP that proposes nothing leaves only the subtrees active in the last step and those
  of point sources to the encode and decode; a subtree whose flow starts in a step is then
  missed, and the fallback runs full steps (judge every 4 steps, miss bound 0);
* where the proposal leaves a subtree out, its leaves that stay dry keep their state in the
  hierarchy (bit for bit where the dry-leaf writer skips them, to the last bit of eta = h + z
  where it writes them), while the wet leaves are still updated;
* (bench.py's learned lines compare the water volume of the learned and plain runs at the
  same simulated time);
* the fused proposal kernel (features from a shared-memory ring, then the MLP) gives the
  proposal of the two-kernel path (features written out, then the MLP) on every tile whose
  ring of coarse cells had activity last step, and proposes nothing elsewhere (both runs
  judge every step, so their states stay identical);
* the device-built feature rows equal the NumPy restatement of the feature builder
  (tests/mlp_ref.py) from the hierarchy, flags and activity bits the previous step left;
* the trainer takes an Adam step on the features and labels a recorded step left on the
  device.
"""
import numpy as np
import pytest

import cases
import mlp_ref
import mwdg2_b200
from gpu_util import FIELDS, assert_same_topology

pytestmark = pytest.mark.gpu
L = 11
STEPS = 6


def _case(tmp_path):
    n = 1 << L
    z = cases.fbm_surface(n, 0.8, 20261203, 30.0)
    h0 = np.maximum(0.0, 10.0 - z)   # valleys filled: many wet leaves from the start
    return cases.fbm_catchment(str(tmp_path), L=L, start_depth=h0, sim_time=600.0)


def _constant_mlp(logit: float) -> np.ndarray:
    p = np.zeros(mwdg2_b200.MLP_PARAMS, np.float32)
    p[-4:] = logit
    return p


def _run(par, setup, steps=STEPS):
    sim = mwdg2_b200.Simulation(par, precision=64)
    setup(sim)
    out = []
    for _ in range(steps):
        sim.step()
        out.append((sim.leaves(), sim.sig(), sim.state(), sim.proposal_stats() if setup is not _none else None))
    sim.close()
    return out


def _none(sim):
    pass


def _same(a, b, what):
    for s, (x, y) in enumerate(zip(a, b)):
        assert_same_topology(x[0], y[0], f"{what} step {s + 1}")
        np.testing.assert_array_equal(x[1], y[1], err_msg=f"{what} step {s + 1}: flags")
        for f in FIELDS:
            np.testing.assert_array_equal(x[2][f], y[2][f], err_msg=f"{what} step {s + 1}: {f}")


def test_recording_and_all_ones_proposal_change_nothing(tmp_path):
    c = _case(tmp_path)
    plain = _run(c.par, _none)
    rec = _run(c.par, lambda s: s.proposal_record(True))
    _same(plain, rec, "recording")
    # with recording on the MLP runs on every coarse cell (the fused kernel would leave out
    # tiles with no activity around them)
    ones = _run(c.par, lambda s: (s.proposal_record(True),
                                  s.proposal_enable(_constant_mlp(20.0), judge_every=0, threshold=0.0, miss_bound=1.0)))
    _same(plain, ones, "all-ones proposal")
    st = ones[-1][3]
    assert st["applied"] == 1.0 and st["proposed"] == st["subtrees"] and st["missed"] == 0
    assert st["active"] > 0 and st["needed"] > 0


def test_empty_proposal_misses_and_falls_back(tmp_path):
    c = _case(tmp_path)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    sim.proposal_enable(_constant_mlp(-20.0), judge_every=4, threshold=0.0, miss_bound=0.0)
    sim.step()                      # the first step always runs in full
    # the MLP proposes nothing: only the subtrees active in the last step and those holding a
    # point source are kept, so a subtree whose flow starts in this step is missed
    missed_at = None
    for s in range(2, 14):
        sim.step()
        st = sim.proposal_stats()
        assert st["proposed"] < st["subtrees"] and st["missed"] <= st["needed"]
        if st["missed"] > 0:   # a judge step (the first after enabling) or an applied one
            missed_at = s
            break
    assert missed_at is not None, "no step left out a subtree that needed it"
    assert st["fallbacks"] == 1 and st["fallback_left"] == 4
    for _ in range(4):
        ok, dt, n = sim.step()
        assert ok and dt > 0
        assert sim.proposal_stats()["applied"] == 0.0
    sim.close()


def _dry_two_rings(sim, tol_h=1e-3) -> np.ndarray:
    """Leaves that are dry, with dry neighbours and dry neighbours' neighbours (the wet test
    of both RK stages of the next step then finds them dry)."""
    lv, st = sim.leaves(), sim.state()
    ids = lv["nb_ids"]
    pos = {int(a): i for i, a in enumerate(lv["act"])}
    dry = st["h0"] < tol_h
    # a neighbour id is a leaf or a significant parent (finer leaves): treat parents as wet
    nb_dry = np.ones(len(dry), bool)
    for d in range(4):
        for i, a in enumerate(ids[d]):
            if a >= 0:
                j = pos.get(int(a))
                nb_dry[i] &= (j is not None) and bool(dry[j])
    one = dry & nb_dry
    two = one.copy()
    for d in range(4):
        for i, a in enumerate(ids[d]):
            if a >= 0:
                j = pos.get(int(a))
                two[i] &= (j is not None) and bool(one[j])
    return two


def test_left_out_dry_subtrees_keep_their_state(tmp_path):
    c = _case(tmp_path)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    sim.proposal_enable(_constant_mlp(-20.0), judge_every=0, threshold=0.0, miss_bound=1.0)
    # the first step runs in full; the next ones keep only the subtrees active in the step
    # before (and those of point sources), and record which leaves stayed dry in both stages
    for _ in range(3):
        sim.step()
    lv = sim.leaves()
    keep = _dry_two_rings(sim) & (lv["lvl"] >= L - 2)
    hier = [[sim.hierarchy(f, m) for m in range(3)] for f in range(3)]
    wet = sim.state()["h0"] >= 1e-3
    sim.step()                      # the dry leaves of left-out subtrees are left as they stand
    stats = sim.proposal_stats()
    assert stats["applied"] == 1.0 and stats["frozen_leaves"] > 0
    lvl = lv["lvl"].astype(np.int64)
    first = ((np.int64(1) << (2 * lvl)) - 1) // 3 + 3
    sub = (lv["act"].astype(np.int64) - first) >> (2 * (lvl - (L - 2)))
    mask = sim.proposal_mask()
    keep &= mask[np.where(keep, sub, 0)] == 0
    assert keep.sum() > 1000
    a = lv["act"][keep]
    # bit for bit where the writer skipped the leaf; where it wrote it (a position that moved,
    # a leaf not dry in both stages of the last step), eta = h + z comes back to the last bit
    for f in range(3):
        for m in range(3):
            e = np.max(np.abs(sim.hierarchy(f, m)[a] - hier[f][m][a]))
            assert e <= 1e-12, f"field {f} mode {m}: {e:.3e}"
    assert np.mean(sim.hierarchy(0, 0)[a] == hier[0][0][a]) > 0.5
    w = lv["act"][wet]
    assert np.any(sim.hierarchy(0, 0)[w] != hier[0][0][w]), "the wet leaves were not updated"
    sim.close()


def test_proposal_keeps_the_water_of_an_inflow(tmp_path):
    """A dry catchment fed by a point inflow, run plain and with an MLP that proposes
    nothing (the subtrees active in the last step and the source's subtree are kept): the
    water volume after 80 steps agrees with the plain run's within 1 %."""
    c = cases.fbm_catchment(str(tmp_path), L=L, sim_time=600.0, peak_q=50.0, t_peak=30.0)
    vols = []
    for learned in (False, True):
        sim = mwdg2_b200.Simulation(c.par, precision=64)
        if learned:
            sim.proposal_enable(_constant_mlp(-20.0), judge_every=0, threshold=0.0, miss_bound=1.0)
        while sim.info()["timestep"] < 80:
            sim.step()
        vols.append((sim.volume(), sim.info()["time"]))
        if learned:
            assert sim.proposal_stats()["learned_steps"] > 70
        sim.close()
    (v0, t0), (v1, t1) = vols
    assert v0 > 0 and abs(v1 - v0) <= 0.01 * v0, f"volume {v1:.6g} m3 at t = {t1:.3f} s, plain {v0:.6g} m3 at {t0:.3f} s"


def test_trainer_observes_a_recorded_step(tmp_path):
    c = _case(tmp_path)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    sim.proposal_record(True)
    sim.step()
    sim.step()
    tr = mwdg2_b200.Trainer(mwdg2_b200.mlp_init(2), lr=1e-3)
    l1 = tr.observe(sim, pos_weight=2.0)
    l2 = tr.observe(sim, pos_weight=2.0)
    assert np.isfinite(l1) and np.isfinite(l2) and l2 < l1
    tr.close()
    sim.close()


def test_features_match_numpy_restatement(tmp_path):
    c = _case(tmp_path)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    sim.proposal_record(True)
    for _ in range(3):
        sim.step()
    hier = [[sim.hierarchy(f, m) for m in range(3)] for f in range(4)]
    sig = sim.sig()
    _, lab_prev = sim.proposal_samples()
    sim.step()
    feats, _ = sim.proposal_samples()
    sim.close()
    want = mlp_ref.proposal_features(hier, sig, L, lab_prev)
    np.testing.assert_array_equal(feats[:, :113], want[:, :113].astype(np.float32))
    assert not np.any(feats[:, 113:])


def _ring_active(labels: np.ndarray, C: int) -> np.ndarray:
    """Per 128-row tile of the coarse level: any activity bit in its 16 x 8 block or ring."""
    nside = 1 << C
    code = np.arange(1 << (2 * C), dtype=np.int64)
    x, y = mlp_ref._compact(code), mlp_ref._compact(code >> 1)
    grid = np.zeros((nside + 2, nside + 2), bool)
    grid[y + 1, x + 1] = labels != 0
    out = np.zeros(len(code) // 128, bool)
    for t in range(len(out)):
        x0, y0 = x[128 * t], y[128 * t]
        out[t] = grid[y0:y0 + 10, x0:x0 + 18].any()
    return out


def test_fused_proposal_matches_two_kernel_path(tmp_path):
    c = _case(tmp_path)
    params = np.load(mwdg2_b200.HERE + "/proposal_mlp.npz")["params"]
    a = mwdg2_b200.Simulation(c.par, precision=64)
    b = mwdg2_b200.Simulation(c.par, precision=64)
    a.proposal_record(True)
    for s in (a, b):
        s.proposal_enable(params, judge_every=1, threshold=-2.0, miss_bound=1.0)
    C = L - 3
    checked = 0
    for step in range(1, 5):
        _, lab_prev = a.proposal_samples() if step > 1 else (None, np.zeros(1 << (2 * C), np.uint8))
        a.step()
        b.step()
        if step == 1:
            continue
        ma, mb = a.proposal_mask(), b.proposal_mask()
        active = np.repeat(_ring_active(lab_prev, C), 512)
        np.testing.assert_array_equal(mb[active], ma[active], err_msg=f"step {step}: active tiles")
        assert not mb[~active].any(), f"step {step}: a tile without activity around it proposed subtrees"
        checked += int(active.sum())
    assert checked > 0
    a.close()
    b.close()
