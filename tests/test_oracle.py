"""CPU tests of the oracle (the C++ restatement of the reference).

The reference cannot be compiled here (no Fortran compiler), so the oracle is
checked against (a) an independent literal Python transliteration of the
routing / depression re-routing routines, (b) known answers of the Numerical
Recipes index sort, and (c) invariants the reference implies: the stack is a
DFS preorder permutation, no local minimum survives LocalMinima, the MFD stack
is a topological order, drainage area and erosion budgets close.
"""
import numpy as np
import pytest

import oracle as O
import fortran_literal as FL
from fastscapelib_fortran import workloads as W


# --------------------------------------------------------------------------
# loc_min_3_indexx

def test_indexx_known_answers():
    # distinct keys: any correct sort gives the unique ascending permutation
    assert list(O.indexx([3.0, 1.0, 2.0])) == [1, 2, 0]
    assert list(O.indexx([5.0])) == [0]
    # 8 elements with ties: traced by hand through the partition step of
    # LocalMinima.f90:985-1040 (median-of-3 puts 2.0 at l as pivot)
    arr = [2.0, 1.0, 2.0, 3.0, 2.0, 1.0, 2.0, 0.0]
    perm = O.indexx(arr)
    lit = [x - 1 for x in FL.indexx(arr)]
    assert list(perm) == lit
    assert list(np.asarray(arr)[perm]) == sorted(arr)


@pytest.mark.parametrize("seed", range(6))
def test_indexx_matches_literal_transliteration(seed):
    rng = np.random.default_rng(seed)
    for n in (1, 2, 7, 8, 9, 31, 64, 257, 1500):
        arr = rng.integers(0, max(2, n // 7), size=n).astype(np.float64)  # heavy ties
        perm = O.indexx(arr)
        lit = np.asarray(FL.indexx(list(arr))) - 1
        assert np.array_equal(perm, lit), (n, seed)
        assert np.all(np.diff(arr[perm]) >= 0)


def test_indexx_distinct_is_argsort():
    rng = np.random.default_rng(7)
    arr = rng.random(5000)
    assert np.array_equal(O.indexx(arr), np.argsort(arr, kind="stable"))


# --------------------------------------------------------------------------
# single-flow routing + LocalMinima against the literal transliteration

CASES = [(21, 17, 1111, 1), (23, 19, 1010, 2), (19, 25, 101, 3), (17, 15, 1000, 4),
         (16, 16, 11, 5), (31, 29, 1111, 6)]


@pytest.mark.parametrize("nx,ny,bc,seed", CASES)
def test_routing_matches_literal(nx, ny, bc, seed):
    wl = W.plain_d8(nx, ny, seed=seed)
    wl.bc = bc
    wl.apply(O)
    O.fastscape_execute_step()
    dx = wl.xl / (nx - 1)
    dy = wl.yl / (ny - 1)
    h_up = wl.h0 + wl.u * wl.dt
    lit = FL.routing_sfd(list(h_up), nx, ny, dx, dy, bc)
    assert np.array_equal(O.copy_int("rec_pre"), np.asarray(lit["rec_pre"]) - 1)
    assert np.array_equal(O.copy_int("stack_pre"), np.asarray(lit["stack_pre"]) - 1)
    d = O.locmin_debug()
    assert d["nbasins"] == lit["nbasins"] and d["basin0"] == lit["basin0"]
    assert np.array_equal(O.copy_int("basins"), np.asarray(lit["basins"]))
    cb = np.asarray(lit["cb"]).reshape(-1, 2)
    cn = np.asarray(lit["cn"]).reshape(-1, 2)
    assert np.array_equal(d["b1"], cb[:, 0]) and np.array_equal(d["b2"], cb[:, 1])
    assert np.array_equal(d["n1"], np.where(cn[:, 0] < 0, -1, cn[:, 0] - 1))
    assert np.array_equal(d["n2"], np.where(cn[:, 1] < 0, -1, cn[:, 1] - 1))
    assert np.array_equal(d["w"], np.asarray(lit["cw"]))
    assert np.array_equal(d["sort_id"], np.asarray(lit["sort_id"]) - 1)
    assert np.array_equal(d["tree"], np.asarray(lit["tree"]) - 1)
    ocb = np.asarray(lit["ocb"]).reshape(-1, 2)
    assert np.array_equal(d["ob1"], ocb[:, 0]) and np.array_equal(d["ob2"], ocb[:, 1])
    assert np.array_equal(O.copy_int("rec"), np.asarray(lit["rec"]) - 1)
    assert np.array_equal(O.copy_int("stack"), np.asarray(lit["stack"]) - 1)
    assert np.array_equal(O.copy_double("length"), np.asarray(lit["length"]))
    assert d["nlocmin_after"] == 0


# --------------------------------------------------------------------------
# invariants over several steps

def _check_stack(stack, rec):
    nn = rec.size
    assert np.array_equal(np.sort(stack), np.arange(nn))
    pos = np.empty(nn, np.int64)
    pos[stack] = np.arange(nn)
    nonroot = rec != np.arange(nn)
    assert np.all(pos[rec[nonroot]] < pos[np.arange(nn)[nonroot]])


@pytest.mark.parametrize("maker", [lambda: W.plain_d8(41, 37, nsteps=5),
                                   lambda: W.mfd(45, 39, nsteps=5),
                                   lambda: W.mfd(33, 47, nsteps=5, n=1.0, bc=101)])
def test_step_invariants(maker):
    wl = maker()
    wl.apply(O)
    nn = wl.nn
    dxdy = (wl.xl / (wl.nx - 1)) * (wl.yl / (wl.ny - 1))
    for step in range(wl.nsteps):
        h_before = O.copy_double("h")
        etot_before = O.copy_double("total_erosion")
        O.fastscape_execute_step()
        assert O.fastscape_get_step() == step + 1
        rec = O.copy_int("rec")
        stack = O.copy_int("stack")
        _check_stack(stack, rec)
        assert O.locmin_debug()["nlocmin_after"] == 0
        a = O.copy_double("drainage_area")
        h = O.copy_double("h")
        if wl.p < -1.5:
            # area = dx*dy*(subtree size), doubled at roots (FlowRouting.f90:136-139)
            size = np.ones(nn)
            for k in stack[::-1]:
                if rec[k] != k:
                    size[rec[k]] += size[k]
            expect = dxdy * size * np.where(rec == np.arange(nn), 2.0, 1.0)
            np.testing.assert_allclose(a, expect, rtol=1e-12)
        else:
            mstack = O.copy_int("mstack")
            mrec = O.copy_slots("mrec")
            mnrec = O.copy_int("mnrec")
            pos = np.empty(nn, np.int64)
            pos[mstack] = np.arange(nn)
            for k in range(nn):
                for t in range(mnrec[k]):
                    assert pos[mrec[k, t]] > pos[k]
            w = O.copy_slots("mwrec")
            sums = np.where(mnrec > 0, w.sum(axis=1), 1.0)
            np.testing.assert_allclose(sums, 1.0, rtol=1e-12)
        # cumulative erosion budget: etot += (h_before + u*dt) - h  (uplift then erosion)
        etot = O.copy_double("total_erosion")
        np.testing.assert_allclose(etot - etot_before, h_before + wl.u * wl.dt - h, atol=1e-8)


def test_setup_errors():
    O.fastscape_init()
    with pytest.raises(RuntimeError, match="nx"):
        O.fastscape_setup()
    O.fastscape_init()
    with pytest.raises(RuntimeError, match="SetUp"):
        O.fastscape_execute_step()
