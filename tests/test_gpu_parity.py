"""GPU parity: the CUDA library (through its C ABI) against the oracle.

Every per-step comparison starts the GPU from the oracle's state (h, b), so
each step is checked on its own.  Tolerances (stated here, checked below):
  * every integer artefact -- receivers, donors, stack, basins, conn list, NR
    sort permutation, MST (Kruskal order), orientation, mrec/mnrec -- is
    bit-exact, single and multiple flow;
  * single flow: float64 fields agree to 1e-12 relative per step.  They are
    not bit-identical only because CUDA's pow and glibc's pow (used by the
    reference through gfortran) may differ in the last ulp;
  * multiple flow: float64 fields agree to 1e-9 relative per step (the
    accumulation also sums donors in a different, equally valid order; the
    multiple-flow stack is a topological order, not the reference's LIFO one);
  * free-running (no re-synchronisation) for 30 steps: h within 1e-7 relative
    L-infinity of the oracle.
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

pytestmark = pytest.mark.gpu

FLOAT_FIELDS = ("h", "drainage_area", "total_erosion", "erosion_rate", "basement", "lake_depth")


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
    g.set_capture(True)
    return g


def gpu_float(g, name):
    out = np.empty(g.nn, np.float64)
    g.copy(name, out)
    return out


def compare_locmin(g, exact=True):
    dg, do = g.locmin_debug(), O.locmin_debug()
    for k in ("nbasins", "basin0", "nconn", "tree_size", "nlocmin_before", "nlocmin_after"):
        assert dg[k] == do[k], (k, dg[k], do[k])
    assert np.array_equal(g.copy_int("basins"), O.copy_int("basins"))
    for k in ("b1", "b2", "n1", "n2", "w", "sort_id", "tree", "ob1", "ob2", "on1", "on2"):
        assert np.array_equal(dg[k], do[k]), k


def compare_routing(g):
    assert np.array_equal(g.copy_int("rec_pre"), O.copy_int("rec_pre"))
    assert np.array_equal(g.copy_int("stack_pre"), O.copy_int("stack_pre"))
    compare_locmin(g)
    assert np.array_equal(g.copy_int("rec"), O.copy_int("rec"))
    assert np.array_equal(g.copy_int("stack"), O.copy_int("stack"))
    nd = g.copy_int("ndon")
    assert np.array_equal(nd, O.copy_int("ndon"))
    dg, do = g.copy_slots("don"), O.copy_slots("don")
    mask = np.arange(8)[None, :] < nd[:, None]
    assert np.array_equal(dg[mask], do[mask])


def rel_err(a, b):
    scale = np.maximum(np.abs(b), 1.0)
    return float(np.max(np.abs(a - b) / scale))


def resync(g):
    """Start the GPU step from the oracle's state."""
    g.set_h(O.copy_double("h"))
    g.set_basement(O.copy_double("basement"))


@pytest.mark.parametrize("nx,ny,bc", [(101, 101, 1111), (64, 48, 1010), (57, 71, 101), (40, 40, 1000)])
def test_sfd_per_step(nx, ny, bc):
    wl = W.plain_d8(nx, ny, seed=nx + ny)
    wl.bc = bc
    wl.apply(O)
    g = make_gpu(wl)
    for step in range(12):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        compare_routing(g)
        assert np.array_equal(gpu_float(g, "length"), O.copy_double("length"))
        for f in ("h", "drainage_area", "erosion_rate", "basement", "lake_depth"):
            a, b = gpu_float(g, f), O.copy_double(f)
            assert rel_err(a, b) <= 1e-12, (step, f, rel_err(a, b))
    assert g.get_step() == O.fastscape_get_step() == 12


@pytest.mark.parametrize("n", [1.0, 1.5])
def test_sfd_newton_per_step(n):
    wl = W.plain_d8(61, 53, seed=5)
    wl.n = n
    wl.apply(O)
    g = make_gpu(wl)
    for _ in range(6):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        compare_routing(g)
        for f in ("h", "drainage_area", "erosion_rate", "lake_depth"):
            a, b = gpu_float(g, f), O.copy_double(f)
            assert rel_err(a, b) <= 1e-12, (f, rel_err(a, b))


@pytest.mark.parametrize("maker", [lambda: W.plain_d8(101, 101, seed=1),
                                   lambda: W.mfd(67, 59, seed=2)])
def test_free_running(maker):
    wl = maker()
    wl.apply(O)
    g = make_gpu(wl)
    for _ in range(30):
        O.fastscape_execute_step()
        g.execute_step()
    err = rel_err(gpu_float(g, "h"), O.copy_double("h"))
    assert err <= 1e-7, err


@pytest.mark.parametrize("nx,ny,bc,n,p", [(65, 65, 1010, 1.5, 1.1), (48, 56, 1111, 1.0, 1.0),
                                           (50, 44, 101, 1.0, -1.0)])
def test_mfd_per_step(nx, ny, bc, n, p):
    wl = W.mfd(nx, ny, seed=nx, n=n, p=p, bc=bc)
    wl.apply(O)
    g = make_gpu(wl)
    for step in range(6):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        compare_routing(g)
        mn = g.copy_int("mnrec")
        assert np.array_equal(mn, O.copy_int("mnrec"))
        mg, mo = g.copy_slots("mrec"), O.copy_slots("mrec")
        mask = np.arange(8)[None, :] < mn[:, None]
        assert np.array_equal(mg[mask], mo[mask])
        wg, wo = g.copy_slots("mwrec"), O.copy_slots("mwrec")
        assert np.max(np.abs(wg[mask] - wo[mask])) <= 1e-12
        for f in ("h", "drainage_area", "erosion_rate", "lake_depth"):
            a, b = gpu_float(g, f), O.copy_double(f)
            assert rel_err(a, b) <= 1e-9, (step, f, rel_err(a, b))
        # the GPU multiple-flow stack is a topological order of mrec
        ms = g.copy_int("mstack")
        pos = np.empty(g.nn, np.int64)
        pos[ms] = np.arange(g.nn)
        rows, cols = np.nonzero(mask)
        assert np.all(pos[mg[rows, cols]] > pos[rows])


def test_reference_api_drop_in():
    """The module-level fastscape_* functions behave like the reference's."""
    import fastscapelib_fortran as fs
    wl = W.plain_d8(51, 45, seed=3)
    wl.apply(fs)
    wl.apply(O)
    for _ in range(3):
        fs.fastscape_execute_step()
        O.fastscape_execute_step()
    hg = np.empty(wl.nn)
    fs.fastscape_copy_h(hg)
    ag = np.zeros((wl.ny, wl.nx))
    fs.fastscape_copy_drainage_area(ag)
    assert rel_err(hg, O.copy_double("h")) <= 1e-12
    assert rel_err(ag.ravel(), O.copy_double("drainage_area")) <= 1e-12
    assert fs.fastscape_get_step() == 3
    with pytest.raises(ValueError):
        fs.fastscape_copy_h(np.empty(wl.nn, np.float32))
    import torch
    ht = torch.empty(wl.nn, dtype=torch.float64, device="cuda")
    fs.fastscape_copy_h(ht)
    assert np.array_equal(ht.cpu().numpy(), hg)  # device copy-out equals host copy-out
    fs.fastscape_destroy()


@pytest.mark.parametrize("precip", ["uniform", "random", "uniform_long_significand"])
def test_sfd_area_is_bit_exact(precip):
    """Single-flow drainage area equals the oracle's bit for bit on both of its
    paths: the closed form v*subtree_size (uniform precipitation, v = dx*dy*P
    with a short significand) and the bottom-up chain sweep (otherwise)."""
    wl = W.plain_d8(83, 71, seed=17)
    wl.apply(O)
    g = make_gpu(wl)
    if precip != "uniform":
        p = (np.random.default_rng(4).random(wl.nn) + 0.5 if precip == "random"
             else np.full(wl.nn, 1.0 / 3.0))
        O.fastscape_set_precip(p)
        g.set_precip(p)
    for _ in range(3):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        assert np.array_equal(gpu_float(g, "drainage_area"), O.copy_double("drainage_area"))
