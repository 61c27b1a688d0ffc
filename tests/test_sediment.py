"""The stream power law with the sediment term (g > 0) on the GPU against the
oracle: Gauss-Seidel iterations with deposition, lake sills, lake water
volumes and the lake-sediment fill (StreamPowerLaw.f90:3-206, 210-400).

Every step starts the GPU from the oracle's h and b.  Checked per step:
  * receivers and stack bit-exact (routing does not depend on g);
  * the number of Gauss-Seidel iterations equal to the oracle's;
  * h, erosion rate, basement and total erosion within 1e-10 relative (single
    flow) and 1e-9 (multiple flow): lake volumes, the multiple-flow erosion
    sum and the convergence measure are summed in another order than the
    reference's stack loops, and CUDA's pow may differ from glibc's in the last
    ulp.
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

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


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def sfd(n, g1, g2, seed):
    wl = W.plain_d8(57, 49, seed=seed)
    wl.n, wl.g1, wl.g2 = n, g1, g2
    wl.kf = np.full(wl.nn, 1e-4)  # strong erosion: sediment to deposit and lakes to fill
    return wl


def mfd(n, p, g1, seed, bc=1010):
    wl = W.mfd(53, 47, seed=seed, n=n, p=p, bc=bc)
    wl.g1 = g1
    wl.kf = np.full(wl.nn, 2e-5)
    return wl


CASES = [("sfd_n1", lambda: sfd(1.0, 1.0, 0.0, 3), 1e-10),
         ("sfd_n15_g2", lambda: sfd(1.5, 0.7, 1.4, 4), 1e-10),
         ("mfd_n1", lambda: mfd(1.0, 1.0, 1.0, 5, bc=1111), 1e-9),
         ("mfd_n15", lambda: mfd(1.5, 1.1, 0.8, 6), 1e-9)]


@pytest.mark.parametrize("name,maker,tol", CASES, ids=[c[0] for c in CASES])
def test_sediment_per_step(name, maker, tol):
    wl = maker()
    wl.apply(O)
    g = make_gpu(wl)
    iters = []
    for step in range(5):
        g.set_h(O.copy_double("h"))
        g.set_basement(O.copy_double("basement"))
        O.fastscape_execute_step()
        g.execute_step()
        assert np.array_equal(g.copy_int("rec"), O.copy_int("rec")), step
        assert np.array_equal(g.copy_int("stack"), O.copy_int("stack")), step
        assert g.gs_iterations() == O.get_ngs(), (step, g.gs_iterations(), O.get_ngs())
        iters.append(O.get_ngs())
        for f in ("h", "erosion_rate", "basement", "total_erosion"):
            a = np.empty(wl.nn)
            g.copy(f, a)
            b = O.copy_double(f)
            assert rel_err(a, b) <= tol, (step, f, rel_err(a, b))
    assert max(iters) > 1, "the case should need more than one Gauss-Seidel iteration"
    g.destroy()


def test_zero_g_takes_the_plain_path():
    wl = W.plain_d8(41, 37, seed=9, nsteps=2)
    g = make_gpu(wl)
    g.execute_step()
    assert g.gs_iterations() == 1
    g.destroy()
