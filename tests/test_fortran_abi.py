"""The reference's own Fortran entry points (gfortran names, every argument by
reference) driven through ctypes, against the oracle.

A program or f2py wrapper built for the reference calls fastscape_init_,
fastscape_set_nx_ny_(&nx, &ny), ..., fastscape_execute_step_(),
fastscape_copy_h_(h) (src/FastScape_api.f90:146-618).  This test makes those
calls on libfsgpu.so exactly so, for a single-flow and a multiple-flow grid,
then compares h, drainage area, erosion rate and the step count with the
oracle after three steps (tolerances of test_gpu_parity: 1e-12 single flow,
1e-9 multiple flow).  Like the reference's `stop`, these entry points end the
process on an error, so the calls run in a child process.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, %(pkg)r); sys.path.insert(0, %(orc)r)
import importlib.util
spec = importlib.util.spec_from_file_location("wl", %(wlp)r)
W = importlib.util.module_from_spec(spec); sys.modules["wl"] = W; spec.loader.exec_module(W)
import oracle as O

lib = ctypes.CDLL(%(lib)r)
P = ctypes.POINTER
ref = ctypes.byref
out = {}
for name, wl in (("sfd", W.plain_d8(53, 47, seed=8)), ("mfd", W.mfd(45, 51, seed=9))):
    keep = []  # arrays passed by pointer stay alive
    def a(x):
        x = np.ascontiguousarray(x, dtype=np.float64); keep.append(x)
        return x.ctypes.data_as(P(ctypes.c_double))
    lib.fastscape_init_()
    lib.fastscape_set_nx_ny_(ref(ctypes.c_int(wl.nx)), ref(ctypes.c_int(wl.ny)))
    lib.fastscape_setup_()
    lib.fastscape_set_xl_yl_(ref(ctypes.c_double(wl.xl)), ref(ctypes.c_double(wl.yl)))
    lib.fastscape_set_dt_(ref(ctypes.c_double(wl.dt)))
    lib.fastscape_init_h_(a(wl.h0.copy()))
    d = lambda v: ref(ctypes.c_double(v))
    lib.fastscape_set_erosional_parameters_(a(wl.kf), d(wl.kfsed), d(wl.m), d(wl.n), a(wl.kd),
                                            d(wl.kdsed), d(wl.g1), d(wl.g2), d(wl.p))
    lib.fastscape_set_u_(a(wl.u))
    lib.fastscape_set_bc_(ref(ctypes.c_int(wl.bc)))
    wl.apply(O)
    for _ in range(3):
        lib.fastscape_execute_step_()
        O.fastscape_execute_step()
    res = {}
    for f, fn in (("h", "fastscape_copy_h_"), ("drainage_area", "fastscape_copy_drainage_area_"),
                  ("erosion_rate", "fastscape_copy_erosion_rate_")):
        buf = np.zeros(wl.nn)
        getattr(lib, fn)(buf.ctypes.data_as(P(ctypes.c_double)))
        r = O.copy_double(f)
        res[f] = float(np.max(np.abs(buf - r) / np.maximum(np.abs(r), 1.0)))
    st = ctypes.c_int(-1)
    lib.fastscape_get_step_(ref(st))
    nx, ny = ctypes.c_int(0), ctypes.c_int(0)
    lib.fastscape_get_sizes_(ref(nx), ref(ny))
    res["step"] = st.value
    res["sizes"] = [nx.value, ny.value]
    lib.fastscape_destroy_()
    out[name] = res
print(json.dumps(out))
"""


def test_fortran_entry_points_by_reference():
    pkg = os.path.join(ROOT, "fastscapelib-fortran_b200")
    code = CHILD % {"pkg": pkg, "orc": os.path.join(ROOT, "oracle"),
                    "wlp": os.path.join(pkg, "fastscapelib_fortran", "workloads.py"),
                    "lib": os.path.join(pkg, "fastscapelib_fortran", "libfsgpu.so")}
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    for name, tol in (("sfd", 1e-12), ("mfd", 1e-9)):
        d = res[name]
        assert d["step"] == 3, d
        for f in ("h", "drainage_area", "erosion_rate"):
            assert d[f] <= tol, (name, f, d)
    assert res["sfd"]["sizes"] == [53, 47] and res["mfd"]["sizes"] == [45, 51]
