"""The mixed-precision form against the FP64 oracle.

Mixed precision (fsb_set_precision(FSB_PREC_MIXED)) keeps the elevation
state, the per-step h update and the ADI residuals in FP64 and integer routing
exact, and runs the multiple-flow weights, the drainage area, the stream-power
erosion factors and Newton iterations (for the increment of h) and the
tridiagonal solves (for the increment of the surface) in FP32.

Stated bounds, relative L-infinity max|x - x_oracle| / max(|x_oracle|, 1):
  * routing (receivers, stack, basins, mrec) identical to the oracle's on
    every step started from the oracle's state (the routing reads the FP64
    state only);
  * per step, started from the oracle's state: the limits in TOL (h 1e-6,
    drainage area 1e-5: FP32 sums along flow paths);
  * free-running: the FP32 differences of each step change receivers at
    near-ties later on, and such a change is carried forward, so a free run
    is bounded loosely (h 1e-4 after 50 steps) -- the same mechanism moves the
    FP64 form away from the oracle over hundreds of steps (test_long_runs.py).
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

from test_gpu_parity import compare_routing, gpu_float, make_gpu, rel_err, resync

pytestmark = pytest.mark.gpu

FIELDS = ("h", "drainage_area", "total_erosion", "erosion_rate", "basement", "lake_depth")
TOL = {"h": 1e-6, "drainage_area": 1e-5, "total_erosion": 1e-6, "erosion_rate": 1e-3,
       "basement": 1e-6, "lake_depth": 1e-6}


def make_mixed(wl):
    g = make_gpu(wl)
    g.set_precision("mixed")
    assert g.get_precision() == "mixed"
    return g


@pytest.mark.parametrize("nx,ny,bc,n,p", [(129, 129, 1010, 1.5, 1.1), (96, 80, 1111, 1.0, 1.0),
                                           (70, 64, 1000, 1.5, 1.1)])
def test_mixed_per_step(nx, ny, bc, n, p):
    wl = W.mfd(nx, ny, seed=nx + 1, n=n, p=p, bc=bc)
    wl.apply(O)
    g = make_mixed(wl)
    for step in range(5):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        compare_routing(g)
        assert np.array_equal(g.copy_int("mnrec"), O.copy_int("mnrec"))
        for f in FIELDS:
            e = rel_err(gpu_float(g, f), O.copy_double(f))
            assert e <= TOL[f], (step, f, e)


@pytest.mark.parametrize("maker", [lambda: W.mfd(129, 129, seed=3, nsteps=50),
                                   lambda: W.plain_d8(101, 101, seed=4, nsteps=50)])
def test_mixed_free_running(maker):
    wl = maker()
    wl.apply(O)
    g = make_mixed(wl)
    for _ in range(wl.nsteps):
        O.fastscape_execute_step()
        g.execute_step()
    e = rel_err(gpu_float(g, "h"), O.copy_double("h"))
    assert e <= 1e-4, e


def test_mixed_and_plain_share_routing():
    """Mixed and FP64 instances of one grid route identically on the first
    step and differ only in floating point afterwards."""
    import fastscapelib_fortran as fs
    wl = W.mfd(97, 89, seed=11, nsteps=1)
    out = {}
    for prec in ("fp64", "mixed"):
        g = fs.FastScape()
        g.set_nx_ny(wl.nx, wl.ny)
        g.setup()
        g.set_precision(prec)
        g.set_xl_yl(wl.xl, wl.yl)
        g.set_dt(wl.dt)
        g.init_h(wl.h0)
        g.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2,
                                   wl.p)
        g.set_u(wl.u)
        g.set_bc(wl.bc)
        g.execute_step()
        out[prec] = (g.copy_int("rec"), g.copy_int("stack"), g.copy_slots("mrec"),
                     gpu_float(g, "h"))
        g.destroy()
    for a, b in zip(out["fp64"][:3], out["mixed"][:3]):
        assert np.array_equal(a, b)
    assert rel_err(out["mixed"][3], out["fp64"][3]) <= 1e-6
