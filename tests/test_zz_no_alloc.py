"""mwdg2_leaf_topology_static: leaf topology for callers that cannot call cudaMalloc.

Those callers (code under a memory manager that owns all device memory, real-time loops
that must not enter the CUDA allocator) pass their own output buffers; the kernels'
scratch lives in a fixed device array inside the library. The tests call the entry point
through the C ABI:

* twice in a row, on two different trees of one simulation, each result against the leaf
  list the simulation itself reports through mwdg2_get_leaves (integers: exact match);
* on random flag trees built on the host at max_ref_lvl 5 (the whole mesh is one tile)
  and 6, with DEMs narrower than the mesh and of unequal sides, against the CPU oracle's
  traversal and compaction of the same flags, on a stream of the caller's own;
* checking that the device's free memory is the same before and after a call.

Device buffers come from torch, which is plumbing here; the entry point takes plain
pointers. This file is collected last, so a run that stops at its first failure has run
every other test before it.
"""
import ctypes
import tempfile

import numpy as np
import pytest

import cases
import mwdg2_b200
import oracle_py

pytestmark = pytest.mark.gpu


def _bind():
    lib = mwdg2_b200.lib()
    f = lib.mwdg2_leaf_topology_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    return f


class _Buffers:
    """Device inputs and outputs of one call, allocated up front by the caller."""

    def __init__(self, torch, sig: np.ndarray, L: int):
        self.cap = 4 ** L
        self.sig = torch.from_numpy(np.ascontiguousarray(sig)).cuda()
        self.act = torch.full((self.cap,), -7, dtype=torch.int32, device="cuda")
        self.lvl = torch.full((self.cap,), 255, dtype=torch.uint8, device="cuda")
        self.ids = torch.full((4 * self.cap,), -7, dtype=torch.int32, device="cuda")
        self.lvls = torch.full((4 * self.cap,), 255, dtype=torch.uint8, device="cuda")

    def call(self, f, L: int, xsz: int, ysz: int, stream=None) -> int:
        n = ctypes.c_int64(-1)
        st = f(self.sig.data_ptr(), L, xsz, ysz, self.act.data_ptr(), self.lvl.data_ptr(), self.ids.data_ptr(),
               self.lvls.data_ptr(), self.cap, ctypes.byref(n), stream)
        assert st == 0, mwdg2_b200.lib().mwdg2_last_error().decode()
        return n.value

    def result(self, k: int) -> dict:
        ids = self.ids.cpu().numpy().reshape(4, self.cap)[:, :k]
        lvls = self.lvls.cpu().numpy().reshape(4, self.cap)[:, :k].astype(np.int32)
        return {"act": self.act.cpu().numpy()[:k], "lvl": self.lvl.cpu().numpy()[:k].astype(np.int32),
                "nb_ids": ids, "nb_lvls": lvls}


def _assert_same(got: dict, want: dict, what: str):
    for key in ("act", "lvl", "nb_ids", "nb_lvls"):
        np.testing.assert_array_equal(got[key], want[key], err_msg=f"{what}: {key}")


def _random_tree(L: int, seed: int, p: float) -> np.ndarray:
    """Significance flags closed upwards (a significant node's parent is significant):
    the root is significant and every child of a significant node is, with probability p."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sig = np.zeros(((1 << (2 * L)) - 1) // 3 + 3, np.uint8)
    sig[3] = 1
    for level in range(1, L):
        first, parent_first = ((1 << (2 * level)) - 1) // 3 + 3, ((1 << (2 * level - 2)) - 1) // 3 + 3
        parents = sig[parent_first:parent_first + (1 << (2 * level - 2))]
        on = np.repeat(parents, 4) & (rng.random(1 << (2 * level)) < p)
        sig[first:first + (1 << (2 * level))] = on
    return sig


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
            buf = _Buffers(torch, sim.sig(), info["L"])
            k = buf.call(f, info["L"], info["xsz"], info["ysz"])
            _assert_same(buf.result(k), want, f"call {call + 1}")
        sim.close()


@pytest.mark.parametrize("L,xsz,ysz,p", [(5, 32, 32, 0.7), (5, 27, 19, 0.85), (6, 64, 41, 0.65), (6, 37, 64, 0.75),
                                         (6, 1, 50, 0.7)])
def test_static_leaf_topology_matches_oracle_on_host_built_trees(L, xsz, ysz, p):
    torch = pytest.importorskip("torch")
    f = _bind()
    stream = torch.cuda.Stream()
    for seed in (1, 2):
        sig = _random_tree(L, 1000 * L + xsz + seed, p)
        want = oracle_py.leaf_topology(sig, L, xsz, ysz)
        buf = _Buffers(torch, sig, L)
        k = buf.call(f, L, xsz, ysz, ctypes.c_void_p(stream.cuda_stream))
        assert k == len(want["act"]), f"L={L} {xsz}x{ysz} seed {seed}: {k} leaves, oracle {len(want['act'])}"
        _assert_same(buf.result(k), want, f"L={L} {xsz}x{ysz} seed {seed}")


def test_static_leaf_topology_leaves_device_memory_untouched():
    torch = pytest.importorskip("torch")
    f = _bind()
    L = 8
    sig = _random_tree(L, 77, 0.7)
    buf = _Buffers(torch, sig, L)
    k1 = buf.call(f, L, 256, 200)   # the first call may load the library's device code
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    k2 = buf.call(f, L, 256, 200)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert k1 == k2
    assert free_after == free_before, f"free device memory changed by {free_before - free_after} bytes"
    _assert_same(buf.result(k2), oracle_py.leaf_topology(sig, L, 256, 200), "second call")


def test_static_leaf_topology_rejects_levels_beyond_its_scratch():
    f = _bind()
    n = ctypes.c_int64(-1)
    dummy = ctypes.c_void_p(16)
    st = f(dummy, 14, 16384, 16384, dummy, dummy, dummy, dummy, 4 ** 14, ctypes.byref(n), None)
    assert st == 6
    assert "max_ref_lvl" in mwdg2_b200.lib().mwdg2_last_error().decode()
