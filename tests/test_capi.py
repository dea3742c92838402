"""The C-ABI library loads and exports every entry point declared in include/mwdg2.h,
and rejects bad input without touching a GPU."""
import ctypes
import os

import pytest

import mwdg2_b200


def test_header_lists_entry_points():
    names = mwdg2_b200.exported_symbols()
    for must in ("mwdg2_create", "mwdg2_step", "mwdg2_run", "mwdg2_run_simulation", "mwdg2_get_leaves",
                 "mwdg2_get_state", "mwdg2_get_sig", "mwdg2_read_stage", "mwdg2_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = mwdg2_b200.lib()
    for name in mwdg2_b200.exported_symbols():
        assert hasattr(lib, name), name


def test_default_opts():
    o = mwdg2_b200.Opts()
    mwdg2_b200.lib().mwdg2_default_opts(ctypes.byref(o))
    assert o.precision == 64 and o.device == -1 and o.epsilon < 0 and o.solver == 0 and o.write_outputs == 1


def test_missing_par_is_io_error(tmp_path):
    with pytest.raises(mwdg2_b200.MWDG2Error) as e:
        mwdg2_b200.Simulation(str(tmp_path / "nope.par"))
    assert e.value.status == 1


def test_bad_precision_is_arg_error(tmp_path):
    with pytest.raises(mwdg2_b200.MWDG2Error) as e:
        mwdg2_b200.Simulation(str(tmp_path / "nope.par"), precision=16)
    assert e.value.status == 6


def test_unsupported_solver_keyword_is_parse_error(tmp_path):
    p = tmp_path / "x.par"
    p.write_text("max_ref_lvl 7\nDEMfile a.dem\n")
    with pytest.raises(mwdg2_b200.MWDG2Error) as e:
        mwdg2_b200.Simulation(str(p))
    assert e.value.status == 2


@pytest.mark.parametrize("level", [5, 15])
def test_max_ref_lvl_outside_6_to_14_is_parse_error(tmp_path, level):
    """Level 15 would overflow the 32-bit slot count of level L + 1 (and not fit in memory)."""
    p = tmp_path / "x.par"
    p.write_text(f"mwdg2\ncuda\nmax_ref_lvl {level}\nepsilon 1e-3\nDEMfile a.dem\n")
    with pytest.raises(mwdg2_b200.MWDG2Error) as e:
        mwdg2_b200.Simulation(str(p))
    assert e.value.status == 2
    assert "max_ref_lvl" in str(e.value)


def test_null_handle_calls_are_rejected():
    lib = mwdg2_b200.lib()
    assert lib.mwdg2_step(None, None, None) == 6
    assert lib.mwdg2_info(None, None, 0) == 6
    assert lib.mwdg2_set_decode_mode(None, 1) == 6


def _static_topology():
    f = mwdg2_b200.lib().mwdg2_leaf_topology_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    return f


@pytest.mark.parametrize("sig_addr, level, cap, needle", [
    (16, 14, 4 ** 14, "max_ref_lvl"),   # beyond the static scratch
    (17, 8, 4 ** 8, "aligned"),         # flags are read four bytes at a time
    (16, 8, 4 ** 8 - 1, "cap"),         # output too small for every finest cell
])
def test_static_topology_argument_errors(sig_addr, level, cap, needle):
    """Argument checks of mwdg2_leaf_topology_static run on the host before any device
    work, so the pointers are never dereferenced."""
    f = _static_topology()
    n = ctypes.c_int64(-1)
    out = ctypes.c_void_p(256)
    st = f(ctypes.c_void_p(sig_addr), level, 1 << level, 1 << level, out, out, out, out, cap, ctypes.byref(n), None)
    assert st == 6
    assert needle in mwdg2_b200.lib().mwdg2_last_error().decode()
    assert n.value == -1


def test_batch_argument_errors(tmp_path):
    """Batch creation checks its arguments and names the failing member; a member whose
    .par is missing fails while reading, before any device work."""
    lib = mwdg2_b200.lib()
    h = ctypes.c_void_p()
    assert lib.mwdg2_batch_create(0, None, None, ctypes.byref(h)) == 6
    missing = str(tmp_path / "nope.par").encode()
    arr = (ctypes.c_char_p * 1)(missing)
    assert lib.mwdg2_batch_create(1, arr, None, ctypes.byref(h)) == 1
    assert "batch member 0" in lib.mwdg2_last_error().decode()
    assert lib.mwdg2_batch_step(None, None, None, None) == 6
    assert lib.mwdg2_batch_member(None, 0, ctypes.byref(h)) == 6
