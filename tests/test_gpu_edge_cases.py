"""GPU parity on the reference's edge cases, through the C ABI, against the oracle.

  * Multiple flow with a free, non-cyclic edge.  find_mult_rec clamps an
    off-grid neighbour onto the edge node and appends it again with the
    diagonal length (FlowRouting.f90:208-226), so a node on such an edge can
    list the same receiver twice with different lengths and weights.  Boundary
    codes 1000 (top edge free, x cyclic), 0010 (bottom edge free, x cyclic),
    1110 (left edge free) and 0111 (bottom edge free, y fixed on top).
  * p = 0: multiple flow with uniform weights, slope**0 = 1
    (FlowRouting.f90:238-242); the literal reading of a "D8 (p=0)" config.
  * A basin graph whose pass heights come nearly in descending order: a
    1025^2 grid falling 0.3 m per row under 1 m of noise.  The reference's NR
    quicksort (LocalMinima.f90:947-1046) degenerates on it to a recursion about
    240 levels deep, which the GPU emulates level by level.

Tolerances as in test_gpu_parity: integer artefacts (receivers, donors, stack,
basins, the basin graph, its sort permutation, Kruskal order, orientation,
mrec/mnrec including duplicate slots) bit-exact; multiple-flow floats within
1e-9 relative per step (summation order of the area differs); mwrec within
1e-12 absolute.
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

from test_gpu_parity import compare_routing, gpu_float, make_gpu, rel_err, resync

pytestmark = pytest.mark.gpu


def compare_mfd_routing(g):
    compare_routing(g)
    mn = g.copy_int("mnrec")
    assert np.array_equal(mn, O.copy_int("mnrec"))
    mask = np.arange(8)[None, :] < mn[:, None]
    mg, mo = g.copy_slots("mrec"), O.copy_slots("mrec")
    assert np.array_equal(mg[mask], mo[mask])
    lg, lo = g.copy_slots("mlrec"), O.copy_slots("mlrec")
    assert np.array_equal(lg[mask], lo[mask])
    wg, wo = g.copy_slots("mwrec"), O.copy_slots("mwrec")
    assert np.max(np.abs(wg[mask] - wo[mask])) <= 1e-12
    return mg, mask


@pytest.mark.parametrize("bc", [1000, 10, 1110, 111])
@pytest.mark.parametrize("p", [1.1, 1.0])
def test_mfd_free_edge_duplicates(bc, p):
    wl = W.mfd(61, 47, seed=bc + 3, n=1.0 if p == 1.0 else 1.5, p=p, bc=bc)
    wl.apply(O)
    g = make_gpu(wl)
    dup_seen = 0
    for step in range(5):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        mg, mask = compare_mfd_routing(g)
        # count nodes that list one receiver in two slots (clamp duplicates)
        rows = np.nonzero(mask.sum(1) > 1)[0]
        for r in rows:
            v = mg[r, mask[r]]
            dup_seen += len(v) != len(np.unique(v))
        for f in ("h", "drainage_area", "erosion_rate", "lake_depth"):
            a, b = gpu_float(g, f), O.copy_double(f)
            assert rel_err(a, b) <= 1e-9, (step, f, rel_err(a, b))
    assert dup_seen > 0, "the free edge produced no duplicate receivers"


@pytest.mark.parametrize("nx,ny,bc", [(101, 101, 1111), (64, 52, 1010)])
def test_mfd_uniform_weights_p0(nx, ny, bc):
    wl = W.plain_d8(nx, ny, seed=nx + 7, p=0.0)
    wl.bc = bc
    wl.apply(O)
    g = make_gpu(wl)
    for step in range(6):
        resync(g)
        O.fastscape_execute_step()
        g.execute_step()
        _, mask = compare_mfd_routing(g)
        wg = g.copy_slots("mwrec")
        mn = g.copy_int("mnrec")
        has = mn > 0
        # uniform weights: every receiver slot of a node carries 1/mnrec
        assert np.allclose(wg[has, 0], 1.0 / mn[has], rtol=0, atol=1e-15)
        for f in ("h", "drainage_area", "erosion_rate", "lake_depth"):
            a, b = gpu_float(g, f), O.copy_double(f)
            assert rel_err(a, b) <= 1e-9, (step, f, rel_err(a, b))


def test_falling_ramp_deep_sort():
    """1025^2, h = U[0,1) - 0.3*row: LocalMinima's basin graph sorted by an NR
    quicksort whose recursion is hundreds of levels deep; every LocalMinima
    artefact bit-exact, floats within 1e-12 (single flow)."""
    nx = 1025
    wl = W.plain_d8(nx, nx, seed=31, nsteps=1)
    j = np.repeat(np.arange(nx, dtype=np.float64), nx)
    wl.h0 = np.random.default_rng(31).random(nx * nx) - 0.3 * j
    wl.apply(O)
    g = make_gpu(wl)
    O.fastscape_execute_step()
    g.execute_step()
    compare_routing(g)
    dbg = O.locmin_debug()
    assert dbg["nconn"] > 100000, dbg["nconn"]
    for f in ("h", "drainage_area", "erosion_rate", "lake_depth"):
        a, b = gpu_float(g, f), O.copy_double(f)
        assert rel_err(a, b) <= 1e-12, (f, rel_err(a, b))
