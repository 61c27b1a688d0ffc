"""Advection (Advect.f90, FastScape_Set_V) on the GPU against the oracle.

  * advection alone (no uplift, no erosion, no diffusion): h, basement and
    total erosion bit-exact -- the x- and y-pass coefficients and the Thomas
    recurrence are the reference's operations in the reference's order;
  * advection inside full steps (single and multiple flow, resynchronised
    each step): within the per-step tolerances of the parity tests (1e-12
    single flow, 1e-9 multiple flow).
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W
from test_oracle import velocity_field

pytestmark = pytest.mark.gpu


def make_gpu(wl):
    import fastscapelib_fortran as fs
    g = fs.FastScape()
    g.set_nx_ny(wl.nx, wl.ny)
    g.setup()
    g.set_xl_yl(wl.xl, wl.yl)
    g.set_dt(wl.dt)
    g.init_h(wl.h0.copy())
    g.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2, wl.p)
    g.set_u(wl.u)
    g.set_bc(wl.bc)
    return g


def field(g, name):
    out = np.empty(g.nn)
    g.copy(name, out)
    return out


def test_advection_alone_is_bit_exact():
    wl = W.plain_d8(67, 45, seed=71)
    wl.kf = np.zeros(wl.nn)
    wl.kd = np.zeros(wl.nn)
    wl.u = np.zeros(wl.nn)
    vx, vy = velocity_field(wl.nx, wl.ny, 8)
    wl.apply(O)
    O.fastscape_set_v(vx, vy)
    g = make_gpu(wl)
    g.set_v(vx, vy)
    for _ in range(3):
        O.fastscape_execute_step()
        g.execute_step()
    for f in ("h", "basement", "total_erosion"):
        assert np.array_equal(field(g, f), O.copy_double(f)), f
    g.destroy()


@pytest.mark.parametrize("maker,tol", [(lambda: W.plain_d8(61, 53, seed=72), 1e-12),
                                       (lambda: W.mfd(47, 59, seed=73), 1e-9)])
def test_advection_in_full_steps(maker, tol):
    wl = maker()
    vx, vy = velocity_field(wl.nx, wl.ny, 9)
    wl.apply(O)
    O.fastscape_set_v(vx, vy)
    g = make_gpu(wl)
    g.set_v(vx, vy)
    for step in range(4):
        g.set_h(O.copy_double("h"))
        g.set_basement(O.copy_double("basement"))
        O.fastscape_execute_step()
        g.execute_step()
        assert np.array_equal(g.copy_int("rec"), O.copy_int("rec"))
        for f in ("h", "basement", "erosion_rate"):
            a, b = field(g, f), O.copy_double(f)
            err = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0))
            assert err <= tol, (step, f, err)
    g.destroy()
