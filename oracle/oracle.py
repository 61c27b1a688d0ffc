"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates fastscapelib-fortran's continental time step on the CPU
(see fastscape_oracle.cpp for the per-routine reference citations).  Only
tests/, the smoke test and the benchmark's cpu_baseline leg use it, as the
checker.  It mirrors the reference's f2py API (src/FastScape_api.f90): the
same ``fastscape_*`` names and argument orders, with numpy float64 arrays.
Node ids in the debug accessors are 0-based (reference value - 1).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfsoracle.so")
_lib = None

_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

DOUBLE_FIELDS = {
    "h": 0, "basement": 1, "total_erosion": 2, "drainage_area": 3, "erosion_rate": 4,
    "lake_depth": 5, "length": 6, "hwater": 7, "sedflux": 8, "catchment": 9,
    "u": 10, "precip": 11, "kf": 12, "kd": 13,
}
INT_FIELDS = {"rec": 0, "ndon": 1, "stack": 2, "mnrec": 3, "mstack": 4, "basins": 5,
              "rec_pre": 6, "stack_pre": 7}


def build() -> str:
    """Compile the oracle shared library (make in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
                os.path.join(_HERE, "fastscape_oracle.cpp")):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.fso_last_error.restype = ctypes.c_char_p
        L.fso_set_nx_ny.argtypes = [ctypes.c_int, ctypes.c_int]
        L.fso_set_xl_yl.argtypes = [ctypes.c_double, ctypes.c_double]
        L.fso_set_dt.argtypes = [ctypes.c_double]
        L.fso_pow15_diag.argtypes = [ctypes.c_int, ctypes.c_void_p]
        L.fso_set_erosional_parameters.argtypes = [
            _F64P, ctypes.c_double, ctypes.c_double, ctypes.c_double, _F64P,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.fso_set_bc.argtypes = [ctypes.c_int]
        for name in ("fso_set_u", "fso_init_h", "fso_set_h", "fso_set_basement", "fso_set_precip"):
            getattr(L, name).argtypes = [_F64P]
        L.fso_copy_double.argtypes = [ctypes.c_int, _F64P]
        L.fso_copy_int.argtypes = [ctypes.c_int, _I32P]
        L.fso_copy_slots.argtypes = [ctypes.c_int, ctypes.c_void_p]
        L.fso_get_step.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.fso_locmin_counts.argtypes = [_I32P]
        L.fso_locmin_arrays.argtypes = [_I32P, _I32P, _I32P, _I32P, _F64P, _I32P, _I32P,
                                        _I32P, _I32P, _I32P, _I32P]
        L.fso_indexx.argtypes = [ctypes.c_int, _F64P, _I32P]
        L.fso_set_v.argtypes = [_F64P, _F64P]
        L.fso_vtk.argtypes = [_F64P, ctypes.c_double, ctypes.c_char_p]
        for name in ("fso_copy_chi", "fso_copy_slope", "fso_copy_curvature", "fso_get_fluxes",
                     "fso_set_all_layers"):
            getattr(L, name).argtypes = [_F64P]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(lib().fso_last_error().decode())


def _nn() -> int:
    return lib().fso_get_nn()


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    if n is not None and a.size < n:
        raise ValueError(f"array of size {a.size} is smaller than nn={n}")
    return a


# ---- the reference API (FastScape_api.f90) --------------------------------
def fastscape_init():
    _check(lib().fso_init())


def fastscape_set_nx_ny(nx, ny):
    _check(lib().fso_set_nx_ny(int(nx), int(ny)))


def fastscape_setup():
    _check(lib().fso_setup())


def fastscape_destroy():
    _check(lib().fso_destroy())


def fastscape_set_xl_yl(xl, yl):
    _check(lib().fso_set_xl_yl(float(xl), float(yl)))


def fastscape_set_dt(dt):
    _check(lib().fso_set_dt(float(dt)))


def fastscape_set_erosional_parameters(kf, kfsed, m, n, kd, kdsed, g1, g2, p):
    nn = _nn()
    _check(lib().fso_set_erosional_parameters(_f64(kf, nn), kfsed, m, n, _f64(kd, nn), kdsed,
                                              g1, g2, p))


def fastscape_set_bc(bc):
    _check(lib().fso_set_bc(int(bc)))


def fastscape_set_u(u):
    _check(lib().fso_set_u(_f64(u, _nn())))


def fastscape_init_h(h):
    _check(lib().fso_init_h(_f64(h, _nn())))


def fastscape_set_h(h):
    _check(lib().fso_set_h(_f64(h, _nn())))


def fastscape_set_basement(b):
    _check(lib().fso_set_basement(_f64(b, _nn())))


def fastscape_set_precip(p):
    _check(lib().fso_set_precip(_f64(p, _nn())))


def fastscape_reset_cumulative_erosion():
    _check(lib().fso_reset_cumulative_erosion())


def fastscape_execute_step():
    _check(lib().fso_execute_step())


def diffusion_only():
    """One ADI diffusion step (Diffusion.f90) on the current state, nothing else."""
    _check(lib().fso_diffusion_only())


def fastscape_get_step() -> int:
    s = ctypes.c_int(0)
    _check(lib().fso_get_step(ctypes.byref(s)))
    return s.value


def copy_double(name: str) -> np.ndarray:
    out = np.empty(_nn(), dtype=np.float64)
    _check(lib().fso_copy_double(DOUBLE_FIELDS[name], out))
    return out


def fastscape_copy_h(buf):
    buf[...] = copy_double("h").reshape(buf.shape)


def fastscape_copy_drainage_area(buf):
    buf[...] = copy_double("drainage_area").reshape(buf.shape)


# ---- debug accessors (0-based node ids) -------------------------------------
def copy_int(name: str) -> np.ndarray:
    out = np.empty(_nn(), dtype=np.int32)
    _check(lib().fso_copy_int(INT_FIELDS[name], out))
    return out


def copy_slots(name: str) -> np.ndarray:
    fid = {"don": 0, "mrec": 1, "mwrec": 2, "mlrec": 3}[name]
    dt = np.int32 if fid < 2 else np.float64
    out = np.empty((_nn(), 8), dtype=dt)
    _check(lib().fso_copy_slots(fid, out.ctypes.data))
    return out


def pow15_diag(on=None) -> dict:
    """Counters of the n = 1.5 power diagnostic (every multiple-flow Newton
    solve repeated with x*sqrt(x) and sqrt(x) for x**1.5 and x**0.5).
    on=True/False starts/stops it (and resets the counters); None reads."""
    out = np.zeros(7, dtype=np.float64)
    lib().fso_pow15_diag(-1 if on is None else int(bool(on)), out.ctypes.data)
    return {"solves": int(out[0]), "iterations": int(out[1]), "iteration_count_differs": int(out[2]),
            "result_differs": int(out[3]), "max_rel_diff": float(out[4]), "max_iterations": int(out[5]),
            "solves_over_20_iterations": int(out[6])}


def locmin_debug() -> dict:
    cnt = np.zeros(6, dtype=np.int32)
    lib().fso_locmin_counts(cnt)
    nb, basin0, nconn, ntree, nbefore, nafter = (int(x) for x in cnt)
    arr = {k: np.zeros(max(nconn, 1), dtype=np.int32) for k in
           ("b1", "b2", "n1", "n2", "sort_id", "ob1", "ob2", "on1", "on2")}
    arr["w"] = np.zeros(max(nconn, 1), dtype=np.float64)
    arr["tree"] = np.zeros(max(ntree, 1), dtype=np.int32)
    lib().fso_locmin_arrays(arr["b1"], arr["b2"], arr["n1"], arr["n2"], arr["w"], arr["sort_id"],
                            arr["tree"], arr["ob1"], arr["ob2"], arr["on1"], arr["on2"])
    out = {k: v[:nconn] for k, v in arr.items() if k != "tree"}
    out["tree"] = arr["tree"][:ntree]
    out.update(nbasins=nb, basin0=basin0, nconn=nconn, tree_size=ntree,
               nlocmin_before=nbefore, nlocmin_after=nafter)
    return out


def indexx(arr) -> np.ndarray:
    """loc_min_3_indexx (LocalMinima.f90:947-1046), 0-based permutation."""
    a = _f64(arr)
    out = np.empty(a.size, dtype=np.int32)
    rc = lib().fso_indexx(a.size, a, out)
    if rc != 0:
        raise RuntimeError("NSTACK too small in loc_min_3_indexx")
    return out


def get_ngs() -> int:
    return lib().fso_get_ngs()


def _derived(fn) -> np.ndarray:
    out = np.empty(_nn(), dtype=np.float64)
    _check(fn(out))
    return out


def fastscape_copy_chi(buf):
    """CopyChi (FastScape_ctx.f90:228-251)."""
    buf[...] = _derived(lib().fso_copy_chi).reshape(buf.shape)


def fastscape_copy_slope(buf):
    """slope (TerrainDerivatives.f90:3-35), in degrees."""
    buf[...] = _derived(lib().fso_copy_slope).reshape(buf.shape)


def fastscape_copy_curvature(buf):
    """curvature (TerrainDerivatives.f90:39-74)."""
    buf[...] = _derived(lib().fso_copy_curvature).reshape(buf.shape)


def fastscape_copy_catchment(buf):
    buf[...] = copy_double("catchment").reshape(buf.shape)


def fastscape_get_fluxes():
    """compute_fluxes (FastScape_ctx.f90:843-886): (tectonic, erosion, boundary)."""
    out = np.zeros(3, dtype=np.float64)
    _check(lib().fso_get_fluxes(out))
    return float(out[0]), float(out[1]), float(out[2])


def fastscape_set_all_layers(dh):
    """SetAllLayers (FastScape_ctx.f90:660-676) without stratigraphy."""
    _check(lib().fso_set_all_layers(_f64(dh, _nn())))


def fastscape_set_v(ux, uy):
    """FastScape_Set_V (api:634 -> ctx:616-632)."""
    _check(lib().fso_set_v(_f64(ux, _nn()), _f64(uy, _nn())))


def fastscape_vtk(fp, vexp, directory="VTK"):
    """Make_VTK (FastScape_ctx.f90:692-777); the directory must exist."""
    _check(lib().fso_vtk(_f64(fp, _nn()), float(vexp), os.fsencode(directory)))
