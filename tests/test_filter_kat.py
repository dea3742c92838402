"""The reference's filter known-answer tests (source/unittests/unit_tests_mra.cu:7-408,
restated as inputs and expected values in tests/golden/filter_kat.json by
tests/golden/make_filter_kat.py from the reference's own filter constants) against this
library's filter functions: the Haar scale and details, the multiwavelet encode (scale
modes and the nine details) and decode (the four children's modes). tests/filter_kat_host.cu
exposes the same templates the CUDA kernels use on the host; it is compiled here with nvcc.
Tolerance relative to max(1, |expected|): 1e-6 in FP64 (the reference's are_reals_equal
bound), 1e-6 in FP32 too (the sums have 12 terms of size ~10)."""
import ctypes
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
KAT = json.load(open(os.path.join(HERE, "golden", "filter_kat.json")))


@pytest.fixture(scope="module")
def kat_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("kat") / "libkat.so")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-x", "cu", "-Xcompiler", "-fPIC", "-shared",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-o", out,
                    os.path.join(HERE, "filter_kat_host.cu")], check=True, timeout=600)
    lib = ctypes.CDLL(out)
    dp = ctypes.POINTER(ctypes.c_double)
    for f, n in (("kat_mw_encode", 3), ("kat_mw_decode", 3), ("kat_hw_encode", 2)):
        getattr(lib, f).argtypes = [ctypes.c_int] + [dp] * n
        getattr(lib, f).restype = None
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _close(actual, expected, what):
    e = np.asarray(expected, np.float64)
    err = np.max(np.abs(np.asarray(actual) - e) / np.maximum(1.0, np.abs(e)))
    assert err <= KAT["tolerance"], f"{what}: {err:.3e}"


@pytest.mark.parametrize("prec", [64, 32])
def test_haar_encode(kat_lib, prec):
    k = KAT["hw_encode"]
    out = np.zeros(4)
    kat_lib.kat_hw_encode(prec, _p(np.array(k["children"], np.float64)), _p(out))
    _close(out, [k["scale"], k["alpha"], k["beta"], k["gamma"]], "haar")


@pytest.mark.parametrize("prec", [64, 32])
def test_multiwavelet_encode(kat_lib, prec):
    k = KAT["mw_encode"]
    s, d = np.zeros(3), np.zeros(9)
    kat_lib.kat_mw_encode(prec, _p(np.array(k["children"], np.float64).ravel()), _p(s), _p(d))
    _close(s, k["scale"], "scale 0/1x/1y")
    _close(d, np.array(k["details"]).ravel(), "details alpha/beta/gamma x 0/1x/1y")


@pytest.mark.parametrize("prec", [64, 32])
def test_multiwavelet_decode(kat_lib, prec):
    k = KAT["mw_decode"]
    c = np.zeros(12)
    kat_lib.kat_mw_decode(prec, _p(np.array(k["scale"], np.float64)), _p(np.array(k["details"], np.float64).ravel()),
                          _p(c))
    _close(c, np.array(k["children"]).ravel(), "children")


def test_multiwavelet_round_trip_fp64(kat_lib):
    """decode(encode(children)) returns the children (the filter bank is orthogonal)."""
    rng = np.random.default_rng(7)
    for _ in range(20):
        ch = rng.uniform(-50.0, 50.0, size=12)
        s, d, back = np.zeros(3), np.zeros(9), np.zeros(12)
        kat_lib.kat_mw_encode(64, _p(ch), _p(s), _p(d))
        kat_lib.kat_mw_decode(64, _p(s), _p(d), _p(back))
        assert np.max(np.abs(back - ch)) <= 1e-12 * 50.0


@pytest.fixture(scope="module")
def oracle_kat_lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("kato") / "libkato.so")
    subprocess.run([gxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", out,
                    os.path.join(HERE, "filter_kat_oracle.cpp")], check=True, timeout=300)
    lib = ctypes.CDLL(out)
    dp = ctypes.POINTER(ctypes.c_double)
    for f, n in (("kat_oracle_mw_encode", 3), ("kat_oracle_mw_decode", 3), ("kat_oracle_hw_encode", 2)):
        getattr(lib, f).argtypes = [dp] * n
        getattr(lib, f).restype = None
    return lib


def test_oracle_filters_pass_the_same_known_answers(oracle_kat_lib):
    """The CPU oracle's filters (compiled as the oracle is: no fused multiply-adds)."""
    k = KAT["hw_encode"]
    out = np.zeros(4)
    oracle_kat_lib.kat_oracle_hw_encode(_p(np.array(k["children"], np.float64)), _p(out))
    _close(out, [k["scale"], k["alpha"], k["beta"], k["gamma"]], "oracle haar")
    k = KAT["mw_encode"]
    s, d = np.zeros(3), np.zeros(9)
    oracle_kat_lib.kat_oracle_mw_encode(_p(np.array(k["children"], np.float64).ravel()), _p(s), _p(d))
    _close(s, k["scale"], "oracle scale")
    _close(d, np.array(k["details"]).ravel(), "oracle details")
    k = KAT["mw_decode"]
    c = np.zeros(12)
    oracle_kat_lib.kat_oracle_mw_decode(_p(np.array(k["scale"], np.float64)),
                                        _p(np.array(k["details"], np.float64).ravel()), _p(c))
    _close(c, np.array(k["children"]).ravel(), "oracle children")
