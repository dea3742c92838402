"""Python binding (ctypes) of the C ABI in include/mwdg2.h.

`Simulation` is the host-side mirror of the reference's run_simulation
(al0vya/gpu-mwdg2 source/run_simulation.cu): it reads the same .par/.dem/.start/.bci/
.bdy/.stage inputs, advances adaptive time steps on the GPU and exposes the leaf grid,
neighbours, significance flags and state for comparison with the reference.

There is no CPU path: constructing a Simulation without the built library or without a
CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from contextlib import contextmanager

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmwdg2_b200.so")
EXE_PATH = os.path.join(HERE, "gpu-mwdg2")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mwdg2.h")

STATUS = {0: "OK", 1: "ERR_IO", 2: "ERR_PARSE", 3: "ERR_CUDA", 4: "ERR_NUMERIC", 5: "ERR_TIMEOUT",
          6: "ERR_ARG", 7: "ERR_STATE", 8: "DONE"}
STATE_ROWS = ("h0", "qx0", "qy0", "z0", "h1x", "qx1x", "qy1x", "z1x", "h1y", "qx1y", "qy1y", "z1y")


class MWDG2Error(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("device", ctypes.c_int), ("epsilon", ctypes.c_double),
                ("solver", ctypes.c_int), ("dirroot", ctypes.c_char_p), ("write_outputs", ctypes.c_int),
                ("verbose", ctypes.c_int)]


_lib = None


def build() -> None:
    """Compile the library and the gpu-mwdg2 executable for sm_100a."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def exported_symbols() -> list[str]:
    """Names of the functions declared in include/mwdg2.h."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(mwdg2_[a-z_]+)\s*\(", text)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run build() (make -C gpu-mwdg2_b200)")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        i32p = ctypes.POINTER(ctypes.c_int32)
        i64p = ctypes.POINTER(ctypes.c_int64)
        dp = ctypes.POINTER(ctypes.c_double)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.mwdg2_default_opts.argtypes = [ctypes.POINTER(Opts)]
        L.mwdg2_last_error.restype = ctypes.c_char_p
        L.mwdg2_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(Opts), ctypes.POINTER(vp)]
        L.mwdg2_step.argtypes = [vp, dp, i64p]
        L.mwdg2_run.argtypes = [vp, ctypes.c_int64, i64p, i64p]
        L.mwdg2_run_simulation.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.mwdg2_info.argtypes = [vp, dp, ctypes.c_int]
        L.mwdg2_get_leaves.argtypes = [vp, i32p, i32p, i32p, i32p, ctypes.c_int64]
        L.mwdg2_get_state.argtypes = [vp, dp, ctypes.c_int64]
        L.mwdg2_get_sig.argtypes = [vp, u8p, ctypes.c_int64]
        L.mwdg2_get_hierarchy.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int64]
        L.mwdg2_read_stage.argtypes = [vp, dp, ctypes.c_int]
        L.mwdg2_last_step_timing.argtypes = [vp, dp, ctypes.c_int]
        L.mwdg2_set_timing.argtypes = [vp, ctypes.c_int]
        L.mwdg2_last_step_counters.argtypes = [vp, i64p, ctypes.c_int]
        L.mwdg2_destroy.argtypes = [vp]
        L.mwdg2_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(Opts),
                                         ctypes.POINTER(vp)]
        L.mwdg2_batch_step.argtypes = [vp, dp, i64p, i32p]
        L.mwdg2_batch_run.argtypes = [vp, ctypes.c_int64, i64p, i64p, i64p]
        L.mwdg2_batch_member.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.mwdg2_batch_group_max_level.argtypes = [vp, ctypes.c_int]
        L.mwdg2_batch_destroy.argtypes = [vp]
        fp = ctypes.POINTER(ctypes.c_float)
        L.mwdg2_mlp_forward.argtypes = [fp, fp, ctypes.c_int, ctypes.c_int64, ctypes.c_float, fp, u8p]
        L.mwdg2_mlp_grad.argtypes = [fp, fp, ctypes.c_int, u8p, ctypes.c_int64, ctypes.c_float, fp, fp]
        L.mwdg2_trainer_create.argtypes = [fp, ctypes.c_float, ctypes.c_int, ctypes.POINTER(vp)]
        L.mwdg2_trainer_step.argtypes = [vp, fp, ctypes.c_int, u8p, ctypes.c_int64, ctypes.c_float, fp]
        L.mwdg2_trainer_observe.argtypes = [vp, vp, ctypes.c_float, fp]
        L.mwdg2_trainer_params.argtypes = [vp, fp]
        L.mwdg2_trainer_destroy.argtypes = [vp]
        L.mwdg2_volume.argtypes = [vp, dp]
        L.mwdg2_volume.restype = ctypes.c_int
        L.mwdg2_set_decode_mode.argtypes = [vp, ctypes.c_int]
        L.mwdg2_set_decode_mode.restype = ctypes.c_int
        L.mwdg2_proposal_record.argtypes = [vp, ctypes.c_int]
        L.mwdg2_proposal_enable.argtypes = [vp, fp, ctypes.c_int, ctypes.c_float, ctypes.c_float]
        L.mwdg2_proposal_stats.argtypes = [vp, dp, ctypes.c_int]
        L.mwdg2_proposal_samples.argtypes = [vp, fp, u8p, ctypes.c_int64, i64p]
        L.mwdg2_proposal_samples.restype = ctypes.c_int
        L.mwdg2_proposal_mask.argtypes = [vp, u8p, ctypes.c_int64, i64p]
        L.mwdg2_proposal_mask.restype = ctypes.c_int
        for name in ("mwdg2_mlp_forward", "mwdg2_mlp_grad", "mwdg2_trainer_create", "mwdg2_trainer_step",
                     "mwdg2_trainer_observe", "mwdg2_trainer_params", "mwdg2_proposal_record", "mwdg2_proposal_enable",
                     "mwdg2_proposal_stats"):
            getattr(L, name).restype = ctypes.c_int
        for name in ("mwdg2_create", "mwdg2_step", "mwdg2_run", "mwdg2_run_simulation", "mwdg2_info",
                     "mwdg2_get_leaves", "mwdg2_get_state", "mwdg2_get_sig", "mwdg2_get_hierarchy",
                     "mwdg2_read_stage", "mwdg2_last_step_timing", "mwdg2_set_timing", "mwdg2_last_step_counters",
                     "mwdg2_batch_create",
                     "mwdg2_batch_step", "mwdg2_batch_run", "mwdg2_batch_member", "mwdg2_batch_group_max_level"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _check(st: int) -> int:
    if st not in (0, 8):
        raise MWDG2Error(st, lib().mwdg2_last_error().decode())
    return st


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


@contextmanager
def _cwd(path):
    old = os.getcwd()
    os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


class Simulation:
    """One adaptive shallow-water simulation on the GPU.

    Relative file names in the .par resolve against the .par's directory (the reference
    resolves them against the working directory; this wrapper changes into the .par's
    directory while reading and while writing outputs)."""

    def __init__(self, par: str, precision: int = 64, epsilon: float | None = None,
                 solver: str | None = None, dirroot: str | None = None, write_outputs: bool = False,
                 device: int = -1, timing: bool | str = False):
        self.par = os.path.abspath(par)
        self.dir = os.path.dirname(self.par)
        o = _opts(precision, epsilon, solver, dirroot, write_outputs, device, timing is True or timing == "phases")
        self._dirroot = o.dirroot
        h = ctypes.c_void_p()
        with _cwd(self.dir):
            _check(lib().mwdg2_create(self.par.encode(), ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._owned = True
        self.precision = precision
        if timing == "step":
            self.set_timing("step")

    @classmethod
    def _view(cls, handle: ctypes.c_void_p, par: str, precision: int, owner) -> "Simulation":
        """A member of a Batch: getters only; the batch owns and steps it."""
        s = cls.__new__(cls)
        s.par, s.dir, s._h, s._owned, s.precision, s._owner = par, os.path.dirname(par), handle, False, precision, owner
        return s

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                lib().mwdg2_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        a = np.zeros(14)
        _check(lib().mwdg2_info(self._h, _p(a, ctypes.c_double), 14))
        keys = ("time", "dt", "timestep", "n_leaves", "L", "xsz", "ysz", "dx", "epsilon", "solver",
                "precision", "sim_time", "n_det", "n_all")
        d = dict(zip(keys, a.tolist()))
        for k in ("timestep", "n_leaves", "L", "xsz", "ysz", "solver", "precision", "n_det", "n_all"):
            d[k] = int(d[k])
        return d

    def step(self) -> tuple[bool, float, int]:
        dt = ctypes.c_double()
        n = ctypes.c_int64()
        st = _check(lib().mwdg2_step(self._h, ctypes.byref(dt), ctypes.byref(n)))
        return st == 0, dt.value, n.value

    def run(self, max_steps: int = 0) -> tuple[int, int]:
        steps = ctypes.c_int64()
        upd = ctypes.c_int64()
        with _cwd(self.dir):
            _check(lib().mwdg2_run(self._h, max_steps, ctypes.byref(steps), ctypes.byref(upd)))
        return steps.value, upd.value

    def leaves(self) -> dict:
        n = self.info()["n_leaves"]
        act = np.zeros(n, np.int32)
        lvl = np.zeros(n, np.int32)
        ids = np.zeros(4 * n, np.int32)
        lvls = np.zeros(4 * n, np.int32)
        _check(lib().mwdg2_get_leaves(self._h, _p(act, ctypes.c_int32), _p(lvl, ctypes.c_int32),
                                      _p(ids, ctypes.c_int32), _p(lvls, ctypes.c_int32), n))
        return {"act": act, "lvl": lvl, "nb_ids": ids.reshape(4, n), "nb_lvls": lvls.reshape(4, n)}

    def state(self) -> dict:
        n = self.info()["n_leaves"]
        out = np.zeros(12 * n)
        _check(lib().mwdg2_get_state(self._h, _p(out, ctypes.c_double), 12 * n))
        out = out.reshape(12, n)
        return {k: out[i] for i, k in enumerate(STATE_ROWS)}

    def sig(self) -> np.ndarray:
        n = self.info()["n_det"]
        out = np.zeros(n, np.uint8)
        _check(lib().mwdg2_get_sig(self._h, _p(out, ctypes.c_uint8), n))
        return out

    def hierarchy(self, field: int, mode: int) -> np.ndarray:
        n = self.info()["n_all"]
        out = np.zeros(n)
        _check(lib().mwdg2_get_hierarchy(self._h, field, mode, _p(out, ctypes.c_double), n))
        return out

    def stage(self, n_points: int) -> np.ndarray:
        out = np.zeros(max(1, n_points))
        _check(lib().mwdg2_read_stage(self._h, _p(out, ctypes.c_double), n_points))
        return out[:n_points]

    def set_timing(self, mode: str | bool):
        """Timing of the following steps (mwdg2_set_timing): "step" (two events around each
        step, no cost to it: last_step_timing()[7]), "phases" or True (events between the
        phases inside the step's graph, ~10 us each: all eight values), None or False (none)."""
        code = {None: 0, False: 0, "step": 1, "phases": 2, True: 2}[mode]
        _check(lib().mwdg2_set_timing(self._h, code))

    def last_step_timing(self) -> np.ndarray:
        out = np.zeros(8)
        _check(lib().mwdg2_last_step_timing(self._h, _p(out, ctypes.c_double), 8))
        return out

    def volume(self) -> float:
        """Water volume of the current state (m^3), an FP64 reduction on the device."""
        v = ctypes.c_double()
        _check(lib().mwdg2_volume(self._h, ctypes.byref(v)))
        return v.value

    def set_decode_mode(self, mode: str):
        """Decode of the following steps (mwdg2_set_decode_mode): "reference" (every
        significant parent decoded, bit for bit the reference's) or "keep" (children of
        encoded parents keep their values; only parents refined this step are decoded)."""
        code = {"reference": 0, "keep": 1}[mode]
        _check(lib().mwdg2_set_decode_mode(self._h, code))

    def proposal_record(self, on: bool = True):
        """Record the proposal's features (step start) and activity labels (step end)."""
        _check(lib().mwdg2_proposal_record(self._h, 1 if on else 0))

    def proposal_enable(self, params, judge_every: int = 20, threshold: float = 0.0, miss_bound: float = 0.01):
        """Let the MLP with `params` choose the subtrees the encode and decode visit (None: off)."""
        if params is None:
            _check(lib().mwdg2_proposal_enable(self._h, None, 0, 0.0, 0.0))
            return
        p = np.ascontiguousarray(params, np.float32)
        self._prop_params = p
        _check(lib().mwdg2_proposal_enable(self._h, _p(p, ctypes.c_float), judge_every, threshold, miss_bound))

    def proposal_samples(self) -> tuple[np.ndarray, np.ndarray]:
        """Features [n][128] and labels [n] of the last recorded step (n coarse cells)."""
        n = ctypes.c_int64()
        lib().mwdg2_proposal_samples(self._h, None, None, 0, ctypes.byref(n))
        feats = np.zeros((n.value, 128), np.float32)
        labels = np.zeros(n.value, np.uint8)
        _check(lib().mwdg2_proposal_samples(self._h, _p(feats, ctypes.c_float), _p(labels, ctypes.c_uint8), n.value,
                                            ctypes.byref(n)))
        return feats, labels

    def proposal_mask(self) -> np.ndarray:
        """The last step's proposal, one byte per child subtree of the coarse level."""
        n = ctypes.c_int64()
        _check(lib().mwdg2_proposal_mask(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.uint8)
        _check(lib().mwdg2_proposal_mask(self._h, _p(out, ctypes.c_uint8), n.value, ctypes.byref(n)))
        return out

    def proposal_stats(self) -> dict:
        a = np.zeros(12)
        _check(lib().mwdg2_proposal_stats(self._h, _p(a, ctypes.c_double), 12))
        keys = ("active", "missed", "proposed", "applied", "subtrees", "learned_steps", "judge_steps", "judge_miss_rate",
                "fallbacks", "fallback_left", "frozen_leaves", "needed")
        return dict(zip(keys, a.tolist()))

    def last_step_counters(self) -> dict:
        out = np.zeros(11, np.int64)
        _check(lib().mwdg2_last_step_counters(self._h, _p(out, ctypes.c_int64), 11))
        return dict(zip(("encoded", "reencoded", "decoded", "leaves", "detail_slots", "launches", "wet_stage1",
                         "wet_stage2", "h2d_bytes", "d2h_bytes", "frozen_leaves"), out.tolist()))


def _opts(precision, epsilon, solver, dirroot, write_outputs, device, timing) -> Opts:
    o = Opts()
    lib().mwdg2_default_opts(ctypes.byref(o))
    o.precision = precision
    o.device = device
    o.epsilon = -1.0 if epsilon is None else float(epsilon)
    o.solver = {None: 0, "hwfv1": 1, "mwdg2": 2}[solver]
    o.dirroot = dirroot.encode() if dirroot else None
    o.write_outputs = 1 if write_outputs else 0
    o.verbose = 2 if timing else 0
    return o


class Batch:
    """An ensemble of independent simulations stepped together (mwdg2_batch_*): one batch
    step enqueues a time step of every unfinished member on its own stream, then waits for
    all of them. Relative names in each .par resolve against that .par's folder."""

    def __init__(self, pars: list[str], precision: int = 64, epsilon: float | None = None,
                 solver: str | None = None, write_outputs: bool = False, device: int = -1, timing: bool = False):
        self.pars = [os.path.abspath(p) for p in pars]
        o = _opts(precision, epsilon, solver, None, write_outputs, device, timing)
        arr = (ctypes.c_char_p * len(self.pars))(*[p.encode() for p in self.pars])
        h = ctypes.c_void_p()
        _check(lib().mwdg2_batch_create(len(self.pars), arr, ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.precision = precision

    def __len__(self):
        return len(self.pars)

    def step(self) -> tuple[int, np.ndarray, np.ndarray]:
        """(members stepped, next dt per member, leaves per member); 0 members when all are done."""
        n = len(self.pars)
        dts = np.zeros(n)
        leaves = np.zeros(n, np.int64)
        k = ctypes.c_int32()
        _check(lib().mwdg2_batch_step(self._h, _p(dts, ctypes.c_double), _p(leaves, ctypes.c_int64), ctypes.byref(k)))
        return k.value, dts, leaves

    def run(self, max_batch_steps: int = 0) -> tuple[int, int, int]:
        """(batch steps, member steps, leaf updates) until every member is done."""
        bs, ms, upd = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().mwdg2_batch_run(self._h, max_batch_steps, ctypes.byref(bs), ctypes.byref(ms), ctypes.byref(upd)))
        return bs.value, ms.value, upd.value

    def group_max_level(self, level: int):
        """Size classes (one launch per kernel for all their members) hold members of at
        most this max_ref_lvl (default 0: none)."""
        _check(lib().mwdg2_batch_group_max_level(self._h, level))

    def member(self, i: int) -> Simulation:
        h = ctypes.c_void_p()
        _check(lib().mwdg2_batch_member(self._h, i, ctypes.byref(h)))
        return Simulation._view(h, self.pars[i], self.precision, self)

    def close(self):
        if getattr(self, "_h", None):
            lib().mwdg2_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- learned refinement proposal
MLP_PARAMS = 16836
MLP_FEATURES = 113


def mlp_init(seed: int = 0) -> np.ndarray:
    """He-initialised parameter block (W1[64][128] b1 W2[64][64] b2 W3[64][64] b3 W4[4][64] b4)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    parts = []
    for fan_out, fan_in in ((64, 128), (64, 64), (64, 64), (4, 64)):
        parts.append(rng.normal(0.0, np.sqrt(2.0 / fan_in), size=fan_out * fan_in))
        parts.append(np.zeros(fan_out))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == MLP_PARAMS
    return p


def mlp_forward(params: np.ndarray, feats: np.ndarray, threshold: float = 0.0) -> tuple[np.ndarray, np.ndarray]:
    """Logits [n][4] and proposal bits [n][4] (logit > threshold) of the tensor-core MLP."""
    params = np.ascontiguousarray(params, np.float32)
    feats = np.ascontiguousarray(feats, np.float32)
    n, nf = feats.shape
    logits = np.zeros((n, 4), np.float32)
    prop = np.zeros((n, 4), np.uint8)
    fp = ctypes.POINTER(ctypes.c_float)
    _check(lib().mwdg2_mlp_forward(_p(params, ctypes.c_float), _p(feats, ctypes.c_float), nf, n, threshold,
                                   _p(logits, ctypes.c_float), _p(prop, ctypes.c_uint8)))
    return logits, prop


def mlp_grad(params: np.ndarray, feats: np.ndarray, labels: np.ndarray, pos_weight: float = 1.0):
    """Gradient of the weighted logistic loss and the loss, from the tensor-core training kernel."""
    params = np.ascontiguousarray(params, np.float32)
    feats = np.ascontiguousarray(feats, np.float32)
    labels = np.ascontiguousarray(labels, np.uint8)
    n, nf = feats.shape
    grad = np.zeros(MLP_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    _check(lib().mwdg2_mlp_grad(_p(params, ctypes.c_float), _p(feats, ctypes.c_float), nf, _p(labels, ctypes.c_uint8), n,
                                pos_weight, _p(grad, ctypes.c_float), _p(loss, ctypes.c_float)))
    return grad, float(loss[0])


class Trainer:
    """Adam on the device for the proposal MLP."""

    def __init__(self, params: np.ndarray, lr: float = 1e-3, device: int = -1):
        params = np.ascontiguousarray(params, np.float32)
        h = ctypes.c_void_p()
        _check(lib().mwdg2_trainer_create(_p(params, ctypes.c_float), lr, device, ctypes.byref(h)))
        self._h = h

    def step(self, feats: np.ndarray, labels: np.ndarray, pos_weight: float = 1.0) -> float:
        feats = np.ascontiguousarray(feats, np.float32)
        labels = np.ascontiguousarray(labels, np.uint8)
        loss = ctypes.c_float()
        _check(lib().mwdg2_trainer_step(self._h, _p(feats, ctypes.c_float), feats.shape[1], _p(labels, ctypes.c_uint8),
                                        feats.shape[0], pos_weight, ctypes.byref(loss)))
        return loss.value

    def observe(self, sim: "Simulation", pos_weight: float = 1.0) -> float:
        loss = ctypes.c_float()
        _check(lib().mwdg2_trainer_observe(self._h, sim._h, pos_weight, ctypes.byref(loss)))
        return loss.value

    def params(self) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, np.float32)
        _check(lib().mwdg2_trainer_params(self._h, _p(out, ctypes.c_float)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().mwdg2_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_simulation(argv: list[str]) -> int:
    """In-process equivalent of the reference's run_simulation(argc, argv)."""
    arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
    return lib().mwdg2_run_simulation(len(argv), arr)
