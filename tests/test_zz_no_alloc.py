"""mwdg2_leaf_topology_static: leaf topology for callers that cannot call cudaMalloc.

Those callers (code under a memory manager that owns all device memory, real-time loops
that must not enter the CUDA allocator) pass their own output buffers; the kernels'
scratch lives in a fixed device array inside the library. This test calls the entry
point through the C ABI twice in a row, on two different trees of one simulation, and
checks each result against the leaf list the simulation itself reports through
mwdg2_get_leaves (integers: exact match). Device buffers come from torch, which is
plumbing here; the entry point takes plain pointers.
"""
import ctypes
import tempfile

import numpy as np
import pytest

import cases
import mwdg2_b200

pytestmark = pytest.mark.gpu


def _bind():
    lib = mwdg2_b200.lib()
    f = lib.mwdg2_leaf_topology_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    return f


def _topology(f, torch, sig: np.ndarray, L: int, xsz: int, ysz: int):
    cap = 4 ** L
    d_sig = torch.from_numpy(sig).cuda()
    act = torch.full((cap,), -7, dtype=torch.int32, device="cuda")
    lvl = torch.full((cap,), 255, dtype=torch.uint8, device="cuda")
    ids = torch.full((4 * cap,), -7, dtype=torch.int32, device="cuda")
    lvls = torch.full((4 * cap,), 255, dtype=torch.uint8, device="cuda")
    n = ctypes.c_int64(-1)
    st = f(d_sig.data_ptr(), L, xsz, ysz, act.data_ptr(), lvl.data_ptr(), ids.data_ptr(), lvls.data_ptr(), cap,
           ctypes.byref(n), None)
    assert st == 0, mwdg2_b200.lib().mwdg2_last_error().decode()
    torch.cuda.synchronize()
    k = n.value
    ids = ids.cpu().numpy().reshape(4, cap)[:, :k]
    lvls = lvls.cpu().numpy().reshape(4, cap)[:, :k].astype(np.int32)
    return {"act": act.cpu().numpy()[:k], "lvl": lvl.cpu().numpy()[:k].astype(np.int32), "nb_ids": ids,
            "nb_lvls": lvls}


def test_static_leaf_topology_matches_simulation_twice():
    torch = pytest.importorskip("torch")
    f = _bind()
    with tempfile.TemporaryDirectory() as d:
        c = cases.circular_dam_break(d, L=8, solver="mwdg2", massint=None)
        sim = mwdg2_b200.Simulation(c.par, precision=64)
        info = sim.info()
        for call, steps in enumerate((3, 25)):
            while sim.info()["timestep"] <= steps:
                sim.step()
            want = sim.leaves()
            got = _topology(f, torch, sim.sig(), info["L"], info["xsz"], info["ysz"])
            for key in ("act", "lvl", "nb_ids", "nb_lvls"):
                np.testing.assert_array_equal(got[key], want[key], err_msg=f"call {call + 1}: {key}")
        sim.close()


def test_static_leaf_topology_rejects_levels_beyond_its_scratch():
    f = _bind()
    n = ctypes.c_int64(-1)
    dummy = ctypes.c_void_p(16)
    st = f(dummy, 14, 16384, 16384, dummy, dummy, dummy, dummy, 4 ** 14, ctypes.byref(n), None)
    assert st == 6
    assert "max_ref_lvl" in mwdg2_b200.lib().mwdg2_last_error().decode()
