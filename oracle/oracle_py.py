"""ctypes binding of the CPU oracle (oracle/liboracle_mwdg2.so).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker and by bench.py's CPU-baseline
leg. The oracle restates the reference algorithm (al0vya/gpu-mwdg2) on the CPU.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from contextlib import contextmanager

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_mwdg2.so")
_lib = None


def build() -> None:
    """Compile the oracle library (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_char_p, ctypes.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_info.argtypes = [vp, dp]
        L.oracle_step.restype = ctypes.c_int
        L.oracle_step.argtypes = [vp, dp, ip]
        L.oracle_get_leaves.argtypes = [vp, ip, ip, ip, ip]
        L.oracle_get_state.argtypes = [vp, dp]
        L.oracle_get_sig.argtypes = [vp, ctypes.POINTER(ctypes.c_ubyte)]
        L.oracle_get_hier.restype = ctypes.c_int
        L.oracle_get_hier.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.oracle_get_maxes.argtypes = [vp, dp]
        L.oracle_num_threads.restype = ctypes.c_int
        L.oracle_set_keep_values.argtypes = [vp, ctypes.c_int]
        L.oracle_leaf_topology.restype = ctypes.c_int
        L.oracle_leaf_topology.argtypes = [ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ip, ip, ip, ip]
        _lib = L
    return _lib


@contextmanager
def _cwd(path):
    old = os.getcwd()
    os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Oracle:
    """One simulation held by the CPU oracle. Relative input names resolve against the
    .par's directory (the reference resolves them against the working directory, so
    the constructor changes into that directory while reading)."""

    STATE_ROWS = ("h0", "qx0", "qy0", "z0", "h1x", "qx1x", "qy1x", "z1x", "h1y", "qx1y", "qy1y", "z1y")

    def __init__(self, par: str, precision: int = 64, epsilon: float | None = None,
                 solver: str | None = None):
        par = os.path.abspath(par)
        err = ctypes.create_string_buffer(512)
        solver_code = {None: 0, "hwfv1": 1, "mwdg2": 2}[solver]
        with _cwd(os.path.dirname(par)):
            h = lib().oracle_create(par.encode(), precision, -1.0 if epsilon is None else float(epsilon),
                                    solver_code, err, 512)
        if not h:
            raise RuntimeError("oracle_create failed: " + err.value.decode())
        self._h = h
        self.precision = precision

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        a = np.zeros(12)
        lib().oracle_info(self._h, _p(a, ctypes.c_double))
        keys = ("L", "xsz", "ysz", "solver", "n_leaves", "timestep", "current_time", "dt", "dx",
                "epsilon", "n_det", "n_all")
        d = dict(zip(keys, a.tolist()))
        for k in ("L", "xsz", "ysz", "solver", "n_leaves", "timestep", "n_det", "n_all"):
            d[k] = int(d[k])
        return d

    def step(self) -> tuple[bool, float, int]:
        dt = ctypes.c_double()
        n = ctypes.c_int()
        r = lib().oracle_step(self._h, ctypes.byref(dt), ctypes.byref(n))
        return bool(r), dt.value, n.value

    def leaves(self) -> dict:
        n = self.info()["n_leaves"]
        act = np.zeros(n, np.int32)
        lvl = np.zeros(n, np.int32)
        ids = np.zeros(4 * n, np.int32)
        lvls = np.zeros(4 * n, np.int32)
        lib().oracle_get_leaves(self._h, _p(act, ctypes.c_int), _p(lvl, ctypes.c_int),
                                _p(ids, ctypes.c_int), _p(lvls, ctypes.c_int))
        return {"act": act, "lvl": lvl, "nb_ids": ids.reshape(4, n), "nb_lvls": lvls.reshape(4, n)}

    def state(self) -> dict:
        n = self.info()["n_leaves"]
        out = np.zeros(12 * n)
        lib().oracle_get_state(self._h, _p(out, ctypes.c_double))
        out = out.reshape(12, n)
        return {k: out[i] for i, k in enumerate(self.STATE_ROWS)}

    def sig(self) -> np.ndarray:
        n = self.info()["n_det"]
        out = np.zeros(n, np.uint8)
        lib().oracle_get_sig(self._h, _p(out, ctypes.c_ubyte))
        return out

    def hier(self, field: int, mode: int) -> np.ndarray | None:
        n = self.info()["n_all"]
        out = np.zeros(n)
        ok = lib().oracle_get_hier(self._h, field, mode, _p(out, ctypes.c_double))
        return out if ok else None

    def set_keep_values(self, on: bool = True):
        """Keep-values decode from the next step on (the library's decode mode 1): the
        children of parents this step's encode visited keep their values; only parents
        refined this step are decoded."""
        lib().oracle_set_keep_values(self._h, 1 if on else 0)

    def maxes(self) -> np.ndarray:
        out = np.zeros(5)
        lib().oracle_get_maxes(self._h, _p(out, ctypes.c_double))
        return out


def leaf_topology(sig: np.ndarray, L: int, xsz: int, ysz: int) -> dict:
    """Leaf list and neighbours (north, east, south, west) of the tree whose significance
    flags are `sig` (get_lvl_idx(L) bytes), as a step's traversal and compaction give them."""
    sig = np.ascontiguousarray(sig, dtype=np.uint8)
    cap = 4 ** L
    act = np.zeros(cap, np.int32)
    lvl = np.zeros(cap, np.int32)
    ids = np.zeros(4 * cap, np.int32)
    lvls = np.zeros(4 * cap, np.int32)
    n = lib().oracle_leaf_topology(_p(sig, ctypes.c_ubyte), L, xsz, ysz, _p(act, ctypes.c_int), _p(lvl, ctypes.c_int),
                                   _p(ids, ctypes.c_int), _p(lvls, ctypes.c_int))
    return {"act": act[:n], "lvl": lvl[:n], "nb_ids": ids.reshape(4, cap)[:, :n],
            "nb_lvls": lvls.reshape(4, cap)[:, :n]}


def num_threads() -> int:
    return int(lib().oracle_num_threads())
