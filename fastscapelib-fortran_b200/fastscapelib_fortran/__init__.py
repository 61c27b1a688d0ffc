"""Drop-in ``fastscapelib_fortran`` for the continental time step on a B200.

This package exposes the reference's Python API -- the f2py module built from
src/FastScape_api.f90 -- with the same routine names and argument orders:

    fastscape_init, fastscape_set_nx_ny, fastscape_setup, fastscape_set_xl_yl,
    fastscape_set_dt, fastscape_set_erosional_parameters, fastscape_set_u,
    fastscape_set_bc, fastscape_init_h, fastscape_execute_step,
    fastscape_copy_h, fastscape_copy_drainage_area, fastscape_get_step, ...

The model state lives in one device arena (a torch uint8 tensor) and every
operation runs as hand-written sm_100a CUDA kernels in ``libfsgpu.so``,
called through its C ABI (include/fastscape_b200.h) with ctypes.  There is no
CPU fallback: importing this package fails if the library is missing and
``fastscape_setup`` fails if no CUDA device is present.

Differences from the reference, by design:
  * errors raise ``RuntimeError`` where the Fortran executes ``stop``;
  * array arguments may also be torch tensors; CUDA tensors are read/written
    on the device without a host round trip;
  * ``FastScape`` objects give independent instances (the reference keeps one
    global model per process; the module-level functions drive a default one).
"""
from __future__ import annotations

import ctypes
import os

# Batches run one CUDA stream per worker; the driver maps streams onto this
# many hardware work queues (default 8), so more queues keep the workers'
# kernels from waiting on each other.  Read when the CUDA context is created,
# i.e. effective when this package is imported before CUDA is first used.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np

try:
    import torch
except ImportError as exc:  # pragma: no cover - torch is part of the runtime
    raise ImportError("fastscapelib_fortran (B200) needs torch for device memory") from exc

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfsgpu.so")
if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build the CUDA library first (make -C {os.path.dirname(_HERE)})")

_lib = ctypes.CDLL(LIB_PATH)

FSB_HOST, FSB_DEVICE = 0, 1
FIELDS = {"h": 0, "basement": 1, "total_erosion": 2, "drainage_area": 3, "erosion_rate": 4,
          "lake_depth": 5, "length": 6, "hwater": 7, "sedflux": 8, "catchment": 9, "u": 10,
          "precip": 11, "kf": 12, "kd": 13}
INT_FIELDS = {"rec": 0, "ndon": 1, "stack": 2, "mnrec": 3, "mstack": 4, "basins": 5,
              "rec_pre": 6, "stack_pre": 7}
SLOT_FIELDS = {"don": 0, "mrec": 1, "mwrec": 2, "mlrec": 3}
# "fp64": every float in FP64, as the reference.  "mixed": FP64 state, h
# update and residuals, exact routing; FP32 weights, area, Newton iterations
# and tridiagonal solves (include/fastscape_b200.h, fsb_set_precision).
PRECISIONS = {"fp64": 0, "mixed": 1}

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double


def _sig(name, *args, res=ctypes.c_int):
    f = getattr(_lib, name)
    f.argtypes = list(args)
    f.restype = res
    return f


_lib.fsb_last_error.restype = ctypes.c_char_p
_sig("fsb_create", ctypes.POINTER(_vp))
_sig("fsb_destroy", _vp)
_sig("fsb_set_nx_ny", _vp, _i, _i)
_sig("fsb_workspace_bytes", _vp, ctypes.POINTER(ctypes.c_size_t))
_sig("fsb_setup", _vp, _vp, ctypes.c_size_t)
_sig("fsb_set_stream", _vp, _vp)
_sig("fsb_set_xl_yl", _vp, _d, _d)
_sig("fsb_set_dt", _vp, _d)
_sig("fsb_set_erosional_parameters", _vp, _vp, _d, _d, _d, _vp, _d, _d, _d, _d, _i)
_sig("fsb_set_bc", _vp, _i)
_sig("fsb_set_precision", _vp, _i)
_sig("fsb_set_concurrency", _vp, _i)
_sig("fsb_get_precision", _vp, ctypes.POINTER(_i))
_sig("fsb_set_v", _vp, _vp, _vp, _i)
for _n in ("fsb_set_u", "fsb_init_h", "fsb_set_h", "fsb_set_basement", "fsb_set_precip"):
    _sig(_n, _vp, _vp, _i)
_sig("fsb_reset_cumulative_erosion", _vp)
_sig("fsb_execute_step", _vp)
_sig("fsb_execute_steps", _vp, _i)
_sig("fsb_get_step", _vp, ctypes.POINTER(_i))
_sig("fsb_get_sizes", _vp, ctypes.POINTER(_i), ctypes.POINTER(_i))
_sig("fsb_copy_field", _vp, _i, _vp, _i)
_sig("fsb_field_device_ptr", _vp, _i, ctypes.POINTER(_vp))
_sig("fsb_copy_int_field", _vp, _i, _vp, _i)
_sig("fsb_copy_slots", _vp, _i, _vp, _i)
_sig("fsb_set_capture", _vp, _i)
_sig("fsb_locmin_counts", _vp, _vp)
_sig("fsb_copy_locmin", _vp, *([_vp] * 11))
_sig("fsb_synchronize", _vp)
for _n in ("fsb_copy_chi", "fsb_copy_slope", "fsb_copy_curvature"):
    _sig(_n, _vp, _vp, _i)
_sig("fsb_get_fluxes", _vp, ctypes.POINTER(_d), ctypes.POINTER(_d), ctypes.POINTER(_d))
_sig("fsb_set_all_layers", _vp, _vp, _i)
_sig("fsb_get_gs_iterations", _vp, ctypes.POINTER(_i))
_sig("fsb_view", _vp)
_sig("fsb_vtk", _vp, _vp, _i, _d, ctypes.c_char_p)
_sig("fsb_debug", _vp)
_sig("fsb_launch_count", _vp, res=ctypes.c_longlong)
_sig("fsb_set_profile", _vp, _i)
_sig("fsb_stage_times", _vp, _vp, _vp, _i, _i)

_sig("fsb_batch_create", ctypes.POINTER(_vp), _i, _i, ctypes.c_size_t)
_sig("fsb_batch_submit", _vp, _vp, ctypes.POINTER(ctypes.c_longlong))
_sig("fsb_batch_wait", _vp, ctypes.c_longlong, ctypes.POINTER(_i), _vp)
_sig("fsb_batch_run", _vp, _vp, _i, _vp, _vp)
_sig("fsb_batch_memory", _vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
     ctypes.POINTER(_i), ctypes.POINTER(_i))
_sig("fsb_batch_destroy", _vp)

STAGES = ("uplift", "receivers", "stack", "local_minima", "lake_fill", "mfd_receivers",
          "drainage_area", "stream_power", "diffusion", "advection",
          # single kernels inside the stages above
          "k_area_sweep", "k_spl_sweep", "k_thomas_rows", "k_thomas_cols", "k_fill_chains")


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(_lib.fsb_last_error().decode())


class FastScape:
    """One continental-step model instance resident on a CUDA device."""

    def __init__(self, device: int | str | torch.device | None = None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   torch.device(device).index or 0)
        h = _vp()
        _check(_lib.fsb_create(ctypes.byref(h)))
        self._h = h
        self._arena = None
        self.nx = self.ny = 0

    # -- lifecycle ---------------------------------------------------------
    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _lib.fsb_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def _stream(self):
        return torch.cuda.current_stream(self.device)

    def set_nx_ny(self, nx: int, ny: int) -> None:
        self.nx, self.ny = int(nx), int(ny)
        _check(_lib.fsb_set_nx_ny(self._h, self.nx, self.ny))

    @property
    def nn(self) -> int:
        return self.nx * self.ny

    def workspace_bytes(self) -> int:
        b = ctypes.c_size_t(0)
        _check(_lib.fsb_workspace_bytes(self._h, ctypes.byref(b)))
        return b.value

    def setup(self) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("fastscape_setup: no CUDA device (this build has no CPU path)")
        nbytes = self.workspace_bytes()
        with torch.cuda.device(self.device):
            self._arena = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            _check(_lib.fsb_set_stream(self._h, self._stream().cuda_stream))
            _check(_lib.fsb_setup(self._h, self._arena.data_ptr(), nbytes))

    def destroy(self) -> None:
        if self._h:
            _lib.fsb_destroy(self._h)
            self._h = None
        self._arena = None

    # -- array marshalling -------------------------------------------------
    def _in(self, a):
        """(pointer, where, keepalive) for an intent(in) node array."""
        if isinstance(a, torch.Tensor):
            t = a.detach().reshape(-1)
            if t.dtype != torch.float64:
                t = t.to(torch.float64)
            if t.is_cuda:
                t = t.to(self.device).contiguous()
                where = FSB_DEVICE
            else:
                t = t.contiguous()
                where = FSB_HOST
            if t.numel() < self.nn:
                raise ValueError(f"array of size {t.numel()} is smaller than nx*ny={self.nn}")
            return t.data_ptr(), where, t
        arr = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if arr.size < self.nn:
            raise ValueError(f"array of size {arr.size} is smaller than nx*ny={self.nn}")
        return arr.ctypes.data, FSB_HOST, arr

    def _out(self, buf, dtype=np.float64, per_node=1):
        """(pointer, where) of an intent(inout) buffer filled in place."""
        n = self.nn * per_node
        if isinstance(buf, torch.Tensor):
            tdt = {np.float64: torch.float64, np.int32: torch.int32}[dtype]
            if buf.dtype != tdt or not buf.is_contiguous() or buf.numel() < n:
                raise ValueError(f"output tensor must be contiguous {tdt} with >= {n} elements")
            return buf.data_ptr(), FSB_DEVICE if buf.is_cuda else FSB_HOST
        if not isinstance(buf, np.ndarray) or buf.dtype != dtype or not buf.flags.c_contiguous \
                or buf.size < n:
            raise ValueError(f"output array must be a C-contiguous {np.dtype(dtype).name} ndarray "
                             f"with >= {n} elements (filled in place)")
        return buf.ctypes.data, FSB_HOST

    # -- setters (FastScape_api.f90) -----------------------------------------
    def set_xl_yl(self, xl: float, yl: float) -> None:
        _check(_lib.fsb_set_xl_yl(self._h, float(xl), float(yl)))

    def set_dt(self, dt: float) -> None:
        _check(_lib.fsb_set_dt(self._h, float(dt)))

    def set_erosional_parameters(self, kf, kfsed, m, n, kd, kdsed, g1, g2, p) -> None:
        pkf, wkf, k1 = self._in(kf)
        pkd, wkd, k2 = self._in(kd)
        if wkf != wkd:
            k1 = self._in(torch.as_tensor(np.asarray(kf, dtype=np.float64)).to(self.device))[2]
            k2 = self._in(torch.as_tensor(np.asarray(kd, dtype=np.float64)).to(self.device))[2]
            pkf, pkd, wkf = k1.data_ptr(), k2.data_ptr(), FSB_DEVICE
        _check(_lib.fsb_set_erosional_parameters(self._h, pkf, float(kfsed), float(m), float(n),
                                                 pkd, float(kdsed), float(g1), float(g2),
                                                 float(p), wkf))
        self._sync_if_device(wkf)

    def set_precision(self, precision: str) -> None:
        """"fp64" (default, the reference's arithmetic) or "mixed"."""
        _check(_lib.fsb_set_precision(self._h, PRECISIONS[precision]))

    def set_concurrency(self, instances: int) -> None:
        """How many instances share the GPU with this one (1: alone).  Above 1,
        the persistent tree sweeps take a quarter of their blocks, leaving SMs
        to the others; results are unchanged.  Batch jobs set this themselves."""
        _check(_lib.fsb_set_concurrency(self._h, int(instances)))

    def get_precision(self) -> str:
        v = _i()
        _check(_lib.fsb_get_precision(self._h, ctypes.byref(v)))
        return {b: a for a, b in PRECISIONS.items()}[v.value]

    def set_bc(self, bc: int) -> None:
        _check(_lib.fsb_set_bc(self._h, int(bc)))

    def _set(self, fn, a) -> None:
        ptr, where, keep = self._in(a)
        _check(fn(self._h, ptr, where))
        self._sync_if_device(where)
        del keep

    def _sync_if_device(self, where):
        if where == FSB_DEVICE:
            self._stream().synchronize()

    def set_u(self, u) -> None:
        self._set(_lib.fsb_set_u, u)

    def set_v(self, vx, vy) -> None:
        """FastScape_Set_V (api:634): advection velocities; switches advection on."""
        px, wx, kx = self._in(vx)
        py, wy, ky = self._in(vy)
        if wx != wy:
            raise ValueError("vx and vy must both be host or both be device arrays")
        _check(_lib.fsb_set_v(self._h, px, py, wx))
        self._sync_if_device(wx)
        del kx, ky

    def init_h(self, h) -> None:
        self._set(_lib.fsb_init_h, h)

    def set_h(self, h) -> None:
        self._set(_lib.fsb_set_h, h)

    def set_basement(self, b) -> None:
        self._set(_lib.fsb_set_basement, b)

    def set_precip(self, p) -> None:
        self._set(_lib.fsb_set_precip, p)

    def reset_cumulative_erosion(self) -> None:
        _check(_lib.fsb_reset_cumulative_erosion(self._h))

    # -- stepping ------------------------------------------------------------
    def execute_step(self, nsteps: int = 1) -> None:
        _check(_lib.fsb_execute_steps(self._h, int(nsteps)))

    def get_step(self) -> int:
        s = _i(0)
        _check(_lib.fsb_get_step(self._h, ctypes.byref(s)))
        return s.value

    def get_sizes(self):
        return self.nx, self.ny

    def synchronize(self) -> None:
        _check(_lib.fsb_synchronize(self._h))

    def launch_count(self) -> int:
        return int(_lib.fsb_launch_count(self._h))

    def set_profile(self, on: bool = True) -> None:
        """Time every stage with CUDA events on the instance's stream."""
        _check(_lib.fsb_set_profile(self._h, 1 if on else 0))

    def stage_times(self, reset: bool = False) -> dict:
        """Accumulated device milliseconds and call counts per stage."""
        ms = np.zeros(len(STAGES), np.float64)
        calls = np.zeros(len(STAGES), np.int64)
        _check(_lib.fsb_stage_times(self._h, ms.ctypes.data, calls.ctypes.data, len(STAGES),
                                    1 if reset else 0))
        return {s: (float(ms[i]), int(calls[i])) for i, s in enumerate(STAGES)}

    # -- copy-outs -------------------------------------------------------------
    def copy(self, name: str, buf) -> None:
        ptr, where = self._out(buf)
        _check(_lib.fsb_copy_field(self._h, FIELDS[name], ptr, where))
        self._sync_if_device(where)

    def _derived(self, fn, buf) -> None:
        dst, where = self._out(buf)
        _check(fn(self._h, dst, where))
        self._sync_if_device(where)

    def copy_chi(self, buf) -> None:
        """FastScape_Copy_Chi (api:379): chi along the last step's stack."""
        self._derived(_lib.fsb_copy_chi, buf)

    def copy_slope(self, buf) -> None:
        """FastScape_Copy_Slope (api:395): slope in degrees."""
        self._derived(_lib.fsb_copy_slope, buf)

    def copy_curvature(self, buf) -> None:
        """FastScape_Copy_Curvature (api:411)."""
        self._derived(_lib.fsb_copy_curvature, buf)

    def get_fluxes(self):
        """FastScape_Get_Fluxes (api:762): (tectonic, erosion, boundary) fluxes."""
        t, e, b = _d(), _d(), _d()
        _check(_lib.fsb_get_fluxes(self._h, ctypes.byref(t), ctypes.byref(e), ctypes.byref(b)))
        return t.value, e.value, b.value

    def set_all_layers(self, dh) -> None:
        """FastScape_Set_All_Layers (api:680): h and basement += dh."""
        self._set(_lib.fsb_set_all_layers, dh)

    def gs_iterations(self) -> int:
        """Gauss-Seidel iterations of the last stream-power call (nGSStreamPowerLaw)."""
        n = _i()
        _check(_lib.fsb_get_gs_iterations(self._h, ctypes.byref(n)))
        return n.value

    def vtk(self, f, vex: float, directory: str | None = None) -> None:
        """FastScape_VTK (api:728): legacy binary VTK files of the surface with
        the scalar field f, in `directory` (default "VTK", as the reference)."""
        ptr, where, keep = self._in(f)
        _check(_lib.fsb_vtk(self._h, ptr, where, float(vex),
                            None if directory is None else os.fsencode(directory)))
        del keep

    def view(self) -> None:
        """FastScape_View (api:188): prints a summary of the instance."""
        _check(_lib.fsb_view(self._h))

    def debug(self) -> None:
        """FastScape_Debug (api:588): prints routing counts and stage times."""
        _check(_lib.fsb_debug(self._h))

    def field(self, name: str) -> torch.Tensor:
        """Zero-copy float64 view of a device field (shape (ny, nx))."""
        p = _vp()
        _check(_lib.fsb_field_device_ptr(self._h, FIELDS[name], ctypes.byref(p)))
        off = p.value - self._arena.data_ptr()
        return self._arena[off:off + 8 * self.nn].view(torch.float64).view(self.ny, self.nx)

    def copy_int(self, name: str) -> np.ndarray:
        out = np.empty(self.nn, dtype=np.int32)
        _check(_lib.fsb_copy_int_field(self._h, INT_FIELDS[name], out.ctypes.data, FSB_HOST))
        return out

    def copy_slots(self, name: str) -> np.ndarray:
        fid = SLOT_FIELDS[name]
        out = np.empty((self.nn, 8), dtype=np.int32 if fid < 2 else np.float64)
        _check(_lib.fsb_copy_slots(self._h, fid, out.ctypes.data, FSB_HOST))
        return out

    def set_capture(self, on: bool = True) -> None:
        _check(_lib.fsb_set_capture(self._h, 1 if on else 0))

    def locmin_debug(self) -> dict:
        cnt = np.zeros(6, dtype=np.int32)
        _check(_lib.fsb_locmin_counts(self._h, cnt.ctypes.data))
        nb, basin0, nconn, ntree, nbefore, nafter = (int(x) for x in cnt)
        a = {k: np.zeros(max(nconn, 1), dtype=np.int32) for k in
             ("b1", "b2", "n1", "n2", "sort_id", "ob1", "ob2", "on1", "on2")}
        a["w"] = np.zeros(max(nconn, 1), dtype=np.float64)
        a["tree"] = np.zeros(max(ntree, 1), dtype=np.int32)
        _check(_lib.fsb_copy_locmin(self._h, *(a[k].ctypes.data for k in
                                               ("b1", "b2", "n1", "n2", "w", "sort_id", "tree",
                                                "ob1", "ob2", "on1", "on2"))))
        out = {k: v[:nconn] for k, v in a.items() if k != "tree"}
        out["tree"] = a["tree"][:ntree]
        out.update(nbasins=nb, basin0=basin0, nconn=nconn, tree_size=ntree,
                   nlocmin_before=nbefore, nlocmin_after=nafter)
        return out


# ---------------------------------------------------------------------------
# Many grids on one device

class _JobRow(ctypes.Structure):
    """fsb_job of include/fastscape_b200.h."""
    _fields_ = [("nx", _i), ("ny", _i), ("bc", _i), ("nsteps", _i),
                ("xl", _d), ("yl", _d), ("dt", _d),
                ("kfsed", _d), ("m", _d), ("n", _d), ("kdsed", _d), ("g1", _d), ("g2", _d),
                ("p", _d),
                ("kf", _vp), ("kd", _vp), ("u", _vp), ("h0", _vp), ("precip", _vp),
                ("h_out", _vp), ("a_out", _vp), ("etot_out", _vp), ("precision", _i)]


def _f64(a, nn, name):
    a = np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (nn,))
                             if np.ndim(a) == 0 else np.asarray(a, dtype=np.float64).reshape(-1))
    if a.size != nn:
        raise ValueError(f"{name} has {a.size} values, the grid has {nn} nodes")
    return np.ascontiguousarray(a)


class Job:
    """One grid of a batch: the sequence init / set_nx_ny / setup / set_xl_yl /
    set_dt / init_h / set_erosional_parameters / set_u / set_precip / set_bc /
    ``nsteps`` x execute_step / copy_h of the reference's API, as one unit of
    work.  Arrays are float64 with nx*ny values (scalars are broadcast).
    After the batch has run it, ``h`` (and ``a`` / ``etot`` when asked for)
    hold the results and ``t_submit``, ``t_start``, ``t_end`` its times."""

    def __init__(self, nx, ny, xl, yl, dt, h0, kf, kd, u, m, n, p, bc=1111, nsteps=1,
                 kfsed=-1.0, kdsed=-1.0, g1=0.0, g2=0.0, precip=None, want_area=False,
                 want_etot=False, precision="fp64"):
        nn = int(nx) * int(ny)
        self.nx, self.ny, self.nsteps, self.bc = int(nx), int(ny), int(nsteps), int(bc)
        self.xl, self.yl, self.dt = float(xl), float(yl), float(dt)
        self.m, self.n, self.p = float(m), float(n), float(p)
        self.kfsed, self.kdsed, self.g1, self.g2 = float(kfsed), float(kdsed), float(g1), float(g2)
        self.h0 = _f64(h0, nn, "h0")
        self.kf = _f64(kf, nn, "kf")
        self.kd = _f64(kd, nn, "kd")
        self.u = _f64(u, nn, "u")
        self.precip = None if precip is None else _f64(precip, nn, "precip")
        self.h = np.empty(nn)
        self.a = np.empty(nn) if want_area else None
        self.etot = np.empty(nn) if want_etot else None
        self.precision = PRECISIONS[precision]
        self.t_submit = self.t_start = self.t_end = float("nan")
        self.status = None

    @property
    def nn(self) -> int:
        return self.nx * self.ny

    def _row(self) -> _JobRow:
        ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        return _JobRow(self.nx, self.ny, self.bc, self.nsteps, self.xl, self.yl, self.dt,
                       self.kfsed, self.m, self.n, self.kdsed, self.g1, self.g2, self.p,
                       ptr(self.kf), ptr(self.kd), ptr(self.u), ptr(self.h0), ptr(self.precip),
                       ptr(self.h), ptr(self.a), ptr(self.etot), self.precision)


class Batch:
    """Runs Jobs concurrently on one CUDA device (``fsb_batch_*``): ``workers``
    threads with one stream each, admission by device memory within
    ``mem_budget`` bytes (0: 90% of the free memory), jobs started in
    submission order.  ``submit`` returns at once; ``wait`` blocks (without
    the GIL) until that job is done; ``run`` does both for a list."""

    def __init__(self, workers: int = 32, mem_budget: int = 0, device: int | None = None):
        dev = torch.cuda.current_device() if device is None else int(device)
        b = _vp()
        _check(_lib.fsb_batch_create(ctypes.byref(b), dev, int(workers), int(mem_budget)))
        self._b = b
        self._jobs: dict[int, Job] = {}

    def submit(self, job: Job) -> int:
        jid = ctypes.c_longlong()
        _check(_lib.fsb_batch_submit(self._b, ctypes.byref(job._row()), ctypes.byref(jid)))
        job.t_submit = float("nan")
        self._jobs[jid.value] = job
        return jid.value

    def wait(self, jid: int) -> Job:
        job = self._jobs.pop(jid)
        st = _i()
        t = np.zeros(3)
        rc = _lib.fsb_batch_wait(self._b, jid, ctypes.byref(st), t.ctypes.data)
        job.status = st.value
        job.t_submit, job.t_start, job.t_end = (float(x) for x in t)
        _check(rc)
        return job

    def run(self, jobs) -> list:
        ids = [self.submit(j) for j in jobs]
        errors = []
        for jid in ids:
            try:
                self.wait(jid)
            except RuntimeError as exc:
                errors.append(str(exc))
        if errors:
            raise RuntimeError(errors[0])
        return list(jobs)

    def memory(self) -> dict:
        used, budget = ctypes.c_size_t(), ctypes.c_size_t()
        running, pending = _i(), _i()
        _check(_lib.fsb_batch_memory(self._b, ctypes.byref(used), ctypes.byref(budget),
                                     ctypes.byref(running), ctypes.byref(pending)))
        return {"in_use": used.value, "budget": budget.value, "running": running.value,
                "pending": pending.value}

    def close(self) -> None:
        if getattr(self, "_b", None):
            for jid in list(self._jobs):
                try:
                    self.wait(jid)
                except RuntimeError:
                    pass
            _lib.fsb_batch_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Module-level API of the reference (one default instance per process)
_default: FastScape | None = None


def _inst() -> FastScape:
    if _default is None:
        raise RuntimeError("fastscape_init has not been called")
    return _default


def fastscape_init():
    """FastScape_Init (api:146)."""
    global _default
    if _default is not None:
        _default.destroy()
    _default = FastScape()


def fastscape_set_nx_ny(nnx, nny):
    _inst().set_nx_ny(nnx, nny)


def fastscape_setup():
    _inst().setup()


def fastscape_destroy():
    global _default
    if _default is not None:
        _default.destroy()
    _default = None


def fastscape_set_xl_yl(xxl, yyl):
    _inst().set_xl_yl(xxl, yyl)


def fastscape_set_dt(dtt):
    _inst().set_dt(dtt)


def fastscape_set_erosional_parameters(kkf, kkfsed, mm, nnn, kkd, kkdsed, gg1, gg2, pp):
    _inst().set_erosional_parameters(kkf, kkfsed, mm, nnn, kkd, kkdsed, gg1, gg2, pp)


def fastscape_set_bc(jbc):
    _inst().set_bc(jbc)


def fastscape_set_u(up):
    _inst().set_u(up)


def fastscape_init_h(hp):
    _inst().init_h(hp)


def fastscape_set_h(hp):
    _inst().set_h(hp)


def fastscape_set_basement(bp):
    _inst().set_basement(bp)


def fastscape_set_precip(precipp):
    _inst().set_precip(precipp)


def fastscape_reset_cumulative_erosion():
    _inst().reset_cumulative_erosion()


def fastscape_execute_step():
    _inst().execute_step()


def fastscape_get_step():
    return _inst().get_step()


def fastscape_get_sizes():
    return _inst().get_sizes()


def fastscape_copy_h(hp):
    _inst().copy("h", hp)


def fastscape_copy_drainage_area(ap):
    _inst().copy("drainage_area", ap)


def fastscape_copy_basement(bp):
    _inst().copy("basement", bp)


def fastscape_copy_total_erosion(etotp):
    _inst().copy("total_erosion", etotp)


def fastscape_copy_erosion_rate(eratep):
    _inst().copy("erosion_rate", eratep)


def fastscape_copy_lake_depth(lp):
    _inst().copy("lake_depth", lp)


def fastscape_copy_chi(chip):
    _inst().copy_chi(chip)


def fastscape_copy_slope(slopep):
    _inst().copy_slope(slopep)


def fastscape_copy_curvature(curvaturep):
    _inst().copy_curvature(curvaturep)


def fastscape_copy_catchment(catchp):
    _inst().copy("catchment", catchp)


def fastscape_get_fluxes():
    """FastScape_Get_Fluxes (api:762); f2py returns the intent(out) scalars."""
    return _inst().get_fluxes()


def fastscape_set_v(ux, uy):
    _inst().set_v(ux, uy)


def fastscape_set_all_layers(dhp):
    _inst().set_all_layers(dhp)


def fastscape_vtk(fp, vexp):
    """FastScape_VTK (api:728); vexp may be a float or a 0-d array."""
    _inst().vtk(fp, float(np.asarray(vexp)))


def fastscape_view():
    _inst().view()


def fastscape_debug():
    _inst().debug()


__all__ = [n for n in dir() if n.startswith("fastscape_")] + ["FastScape", "Job", "Batch", "LIB_PATH"]
