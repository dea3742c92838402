"""The CPU oracle against the reference build's per-step digests (CPU only).

tests/golden/digest_*.npz hold per-step digests of the leaf list, neighbours and
significance flags written by the reference's own CUDA build (tests/golden/
make_golden_digest.py). The oracle (the reference algorithm restated in C++, FP64, no
fused multiply-adds) reproduces them bit for bit over the whole 3.5 s of the 256^2
circular dam break (292 steps) and over the first 25 steps of the 4096^2 benchmark
catchment (MWDG2).

Not pinned here: HWFV1 on the catchment at max_ref_lvl 12, where the unfused oracle leaves
the reference build at step 1 (about 2000 of 5.6 M parents whose Haar detail norms sit
within rounding of their thresholds on the 3-decimal DEM decide differently); the same
oracle compiled with fused multiply-adds matches all 25 steps. The CUDA product is held
to those fixtures directly (tests/test_gpu_reference_digests.py); FP32 runs are held to
their own FP32 reference build there, since an unfused FP32 oracle parts from it after
about 140 steps of the dam break.
"""
import os
import tempfile

import numpy as np
import pytest

import make_golden_digest as mgd
import oracle_py

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _oracle_digests(dig, o) -> dict:
    lv = o.leaves()
    out = {"leaf_act": dig(lv["act"]), "leaf_lvl": dig(lv["lvl"]), "sig": dig(o.sig(), 8)}
    for k, d in enumerate("nesw"):
        out[f"nb_{d}_ids"] = dig(lv["nb_ids"][k])
        out[f"nb_{d}_lvls"] = dig(lv["nb_lvls"][k])
    return out


@pytest.mark.parametrize("name", ["cdb_mw_l8_fp64_full", "catch_mw_l12_fp64"])
def test_oracle_matches_reference_digests(name):
    spec = mgd.case_specs()[name]
    g = np.load(os.path.join(GOLDEN, f"digest_{name}.npz"))
    names = [str(n) for n in g["names"]]
    present = g["present"]
    dig = mgd.Digester()
    with tempfile.TemporaryDirectory() as d:
        c = mgd.make_case(spec, d)
        o = oracle_py.Oracle(c.par, spec["precision"])
        try:
            for s in range(1, g["digest"].shape[0] + 1):
                ok, dt, n = o.step()
                assert ok and n == int(g["steps_n"][s - 1]), f"{name} step {s}: {n} leaves"
                mine = _oracle_digests(dig, o)
                bad = [k for i, k in enumerate(names) if present[i] and mine[k] != int(g["digest"][s - 1, i])]
                assert not bad, f"{name} step {s}: the oracle differs from the reference build in {bad}"
                assert abs(dt - g["steps_dt"][s - 1]) <= 1e-9 * g["steps_dt"][s - 1]
        finally:
            o.close()


def test_digest_matches_the_hooks_function():
    """The numpy digest is the hooks' function: n * 0x9E3779B97F4A7C15 + sum_i (bits_i + 1) *
    (splitmix64(i) | 1) mod 2^64, checked here against a direct evaluation in Python integers."""
    rng = np.random.Generator(np.random.PCG64(5))
    a = rng.integers(-2 ** 31, 2 ** 31, size=257, dtype=np.int64).astype(np.int32)
    b = rng.integers(0, 2, size=300).astype(np.uint8)
    M = 2 ** 64

    def sm(x):
        x = (x + 0x9E3779B97F4A7C15) % M
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) % M
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) % M
        return x ^ (x >> 31)

    def ref(vals, mask):
        h = (len(vals) * 0x9E3779B97F4A7C15) % M
        for i, v in enumerate(vals):
            h = (h + ((int(v) & mask) + 1) * (sm(i) | 1)) % M
        return h

    dig = mgd.Digester()
    assert dig(a) == ref(a, 0xFFFFFFFF)
    assert dig(b, 8) == ref(b, 0xFF)
    c = a.copy()
    c[100] ^= 1
    assert dig(c) != dig(a)
