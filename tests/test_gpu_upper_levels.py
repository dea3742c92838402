"""The tree levels above the bands (10 and up) against the oracle at max_ref_lvl 12.

The parity cases run at max_ref_lvl 7, where every level is walked by the band kernels;
only larger trees reach the per-level kernels: the dense encode / decode / re-encode
(k_encode_level, k_decode_level), the sparse form of a level with few significant parents
(k_level_sparse), the flags-only extra-significance pass (k_extra_sig_level, levels 10 to
L - 2) and the value decode of those levels on its own stream beside the leaf topology.
This runs the benchmark's 4096^2 fBm catchment (FP64, the reference's leaf order and
neighbour rule) for four steps: the first step sweeps every level; the later ones replay
the captured step, with level 11 in its sparse form once the first step has shown that
fewer than one in eight of its parents are significant. Every step: the significance
flags, leaf list, levels and neighbour ids bit-exact, the state within 1e-10 relative to
max(1, |value|), dt within 1e-9."""
import numpy as np
import pytest

import cases
import mwdg2_b200
import oracle_py
from gpu_util import FIELDS, assert_same_topology, rel_err

pytestmark = pytest.mark.gpu
L = 12
STEPS = 4


def _level(sig: np.ndarray, level: int) -> np.ndarray:
    first = ((1 << (2 * level)) - 1) // 3 + 3
    return sig[first:first + (1 << (2 * level))]


def test_upper_levels_match_oracle_at_level_12(tmp_path):
    c = cases.fbm_catchment(str(tmp_path), L=L)
    sim = mwdg2_b200.Simulation(c.par, precision=64)
    orc = oracle_py.Oracle(c.par, 64)
    try:
        for s in range(1, STEPS + 1):
            ok, dt, n = sim.step()
            ok2, dt2, n2 = orc.step()
            assert ok and ok2 and n == n2, f"step {s}: leaves {n} vs {n2}"
            sig = sim.sig()
            np.testing.assert_array_equal(sig, orc.sig(), err_msg=f"step {s}: significance flags")
            assert_same_topology(sim.leaves(), orc.leaves(), f"step {s}")
            st, so = sim.state(), orc.state()
            for f in FIELDS:
                e = rel_err(st[f], so[f])
                assert e <= 1e-10, f"step {s} {f}: {e:.3e}"
            assert abs(dt - dt2) <= 1e-9 * dt2, f"step {s}: dt {dt} vs {dt2}"
            # the upper levels are really exercised: level 10 dense, level 11 sparse
            l10, l11 = _level(sig, 10), _level(sig, 11)
            assert 8 * int(l10.sum()) >= l10.size, f"step {s}: level 10 should be dense"
            assert 0 < 8 * int(l11.sum()) < l11.size, f"step {s}: level 11 should be sparse"
    finally:
        orc.close()
        sim.close()
