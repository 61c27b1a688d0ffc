"""The rest of the reference's API on the GPU, against the oracle.

Each case steps the GPU and the oracle from the same state (the GPU is given
the oracle's h and b before the last step), then compares:
  * catchment labels: bit-exact (same catch0 stream, bit-exact routing);
  * chi: within 1e-10 relative (a per step is within 1e-12 / 1e-9 of the
    oracle, and pow(a0/a, m/n) differs in the last ulp between CUDA and glibc);
  * slope and curvature of the same h: within 1e-12 relative (slope) and
    1e-10 of the largest |curvature| (atan, sqrt and pow ulps);
  * get_fluxes: within 1e-12 relative (single flow) and 1e-9 (multiple flow),
    the erosion flux relative to the sum of |erate| (erate has both signs);
  * set_all_layers: bit-exact (one addition per node);
  * view and debug print their summaries.
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

pytestmark = pytest.mark.gpu

CASES = [("sfd", lambda: W.plain_d8(45, 39, seed=41, nsteps=3), 1e-12),
         ("sfd_newton", lambda: W.uneven_d8(1, seed=44, nsteps=3, lo=41, hi=41)[0], 1e-12),
         ("mfd", lambda: W.mfd(43, 37, seed=42, nsteps=3), 1e-9),
         ("mfd_bc0101", lambda: W.mfd(37, 41, seed=43, nsteps=3, bc=101, n=1.0, p=1.0), 1e-9)]


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


def rel(x, ref):
    return np.max(np.abs(x - ref) / np.maximum(np.abs(ref), 1.0))


@pytest.mark.parametrize("name,maker,tol", CASES, ids=[c[0] for c in CASES])
def test_derived_fields(name, maker, tol):
    wl = maker()
    g = make_gpu(wl)
    wl.apply(O)
    for _ in range(wl.nsteps - 1):
        O.fastscape_execute_step()
    g.set_h(O.copy_double("h"))
    g.set_basement(O.copy_double("basement"))
    g.execute_step()
    O.fastscape_execute_step()
    nn = wl.nn
    got, ref = np.empty(nn), np.empty(nn)

    g.copy("catchment", got)
    O.fastscape_copy_catchment(ref)
    assert np.array_equal(got, ref)

    g.copy_chi(got)
    O.fastscape_copy_chi(ref)
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) <= max(tol, 1e-10)
    assert np.array_equal(got == 0, ref == 0)

    t, e, b = g.get_fluxes()
    to, eo, bo = O.fastscape_get_fluxes()
    assert abs(t - to) <= 1e-12 * abs(to)
    surf = wl.xl * wl.yl / (wl.nx - 1) / (wl.ny - 1)
    scale = np.abs(O.copy_double("erosion_rate")).sum() * surf  # erate has both signs
    assert abs(e - eo) <= tol * scale
    assert abs(b - bo) <= tol * max(abs(bo), 1e-300)

    h = O.copy_double("h")
    g.set_h(h)
    g.copy_slope(got)
    O.fastscape_copy_slope(ref)
    assert rel(got, ref) <= 1e-12
    g.copy_curvature(got)
    O.fastscape_copy_curvature(ref)
    assert np.max(np.abs(got - ref)) <= 1e-10 * np.abs(ref).max()

    g.set_basement(O.copy_double("basement"))  # same h and b on both sides
    dh = np.random.default_rng(5).standard_normal(nn)
    O.fastscape_set_all_layers(dh)
    g.set_all_layers(dh)
    g.copy("h", got)
    assert np.array_equal(got, O.copy_double("h"))
    g.copy("basement", got)
    assert np.array_equal(got, O.copy_double("basement"))
    g.destroy()


def test_view_debug_and_module_functions(capfd):
    import fastscapelib_fortran as fs
    wl = W.plain_d8(33, 31, seed=3, nsteps=2)
    wl.apply(fs)
    for _ in range(wl.nsteps):
        fs.fastscape_execute_step()
    fs.fastscape_view()
    fs.fastscape_debug()
    out = capfd.readouterr().out
    assert "nx,ny 33 31" in out and "step 2" in out
    assert "Total number of local minima" in out and "Number of nil elements in stack 0" in out
    buf = np.empty(wl.nn)
    for f in (fs.fastscape_copy_chi, fs.fastscape_copy_slope, fs.fastscape_copy_curvature,
              fs.fastscape_copy_catchment):
        f(buf)
        assert np.all(np.isfinite(buf))
    t, e, b = fs.fastscape_get_fluxes()
    assert t > 0 and e > 0 and b > 0
    fs.fastscape_set_all_layers(np.zeros(wl.nn))
