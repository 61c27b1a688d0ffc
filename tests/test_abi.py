"""CPU checks of the C-ABI shared library: it loads without a GPU and exports
every entry point include/fastscape_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fastscape_b200.h")
LIB = os.path.join(ROOT, "fastscapelib-fortran_b200", "fastscapelib_fortran", "libfsgpu.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(fsb_[a-z0-9_]+|fastscape_[a-z0-9_]+_)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "fsb_execute_step" in names and "fastscape_execute_step_" in names
    assert len(names) > 40


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} not built")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_package_imports_without_gpu():
    import fastscapelib_fortran as fs
    assert os.path.samefile(fs.LIB_PATH, LIB)
    for name in ("fastscape_init", "fastscape_setup", "fastscape_set_nx_ny", "fastscape_set_xl_yl",
                 "fastscape_set_dt", "fastscape_set_erosional_parameters", "fastscape_set_u",
                 "fastscape_set_bc", "fastscape_init_h", "fastscape_execute_step",
                 "fastscape_copy_h", "fastscape_copy_drainage_area", "fastscape_get_step",
                 "fastscape_destroy"):
        assert callable(getattr(fs, name))


def test_handle_errors_without_setup():
    import fastscapelib_fortran as fs
    inst = fs.FastScape.__new__(fs.FastScape)
    h = ctypes.c_void_p()
    assert fs._lib.fsb_create(ctypes.byref(h)) == 0
    assert fs._lib.fsb_execute_step(h) != 0
    assert b"SetUp" in fs._lib.fsb_last_error()
    assert fs._lib.fsb_set_nx_ny(h, 2, 2) == 0
    size = ctypes.c_size_t()
    assert fs._lib.fsb_workspace_bytes(h, ctypes.byref(size)) != 0  # nx, ny >= 3 required
    assert fs._lib.fsb_destroy(h) == 0
    del inst


def test_instance_settings_without_gpu():
    """Precision and concurrency are host-side settings of a handle: valid values
    are taken, invalid ones refused with a message."""
    import fastscapelib_fortran as fs
    h = ctypes.c_void_p()
    assert fs._lib.fsb_create(ctypes.byref(h)) == 0
    prec = ctypes.c_int(-1)
    assert fs._lib.fsb_set_precision(h, 1) == 0
    assert fs._lib.fsb_get_precision(h, ctypes.byref(prec)) == 0 and prec.value == 1
    assert fs._lib.fsb_set_precision(h, 7) != 0
    assert b"precision" in fs._lib.fsb_last_error()
    assert fs._lib.fsb_set_concurrency(h, 32) == 0
    assert fs._lib.fsb_set_concurrency(h, 1) == 0
    assert fs._lib.fsb_set_concurrency(h, 0) != 0
    assert b"instances" in fs._lib.fsb_last_error()
    assert fs._lib.fsb_destroy(h) == 0
