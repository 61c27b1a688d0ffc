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
         (16, 16, 11, 5), (31, 29, 1111, 6),
         # the smallest grids: one interior node, one interior row, one interior column
         (3, 3, 1111, 7), (3, 4, 1010, 8), (5, 3, 101, 9), (4, 3, 1000, 10)]


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
    # the lake fill and the drainage area on the re-routed forest
    nn = nx * ny
    h1 = [0.0] + list(h_up)
    hw = FL.lake_fill_sfd(h1, lit["rec_1b"], lit["stack_1b"], nn)
    assert O.copy_double("hwater").tolist() == hw[1:]
    assert O.copy_double("lake_depth").tolist() == [hw[k] - h1[k] for k in range(1, nn + 1)]
    a = FL.flow_accumulation_sfd(lit["stack_1b"], lit["rec_1b"], [0.0] + [1.0] * nn, nn, dx, dy)
    assert O.copy_double("drainage_area").tolist() == a[1:]


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


def _literal_chi(stack, rec, a, length, a0, mn):
    """CopyChi (FastScape_ctx.f90:228-251), loop for loop (0-based ids)."""
    chi = np.zeros(a.size)
    for ijk in stack:
        if a[ijk] > a0:
            chi[ijk] = chi[rec[ijk]] + (a0 / a[ijk]) ** mn * length[ijk]
    return chi


def _literal_slope_curv(h, nx, ny, dx, dy):
    """slope and curvature (TerrainDerivatives.f90:3-74) in plain Python."""
    con = 45.0 / np.arctan(1.0)
    s = np.zeros(nx * ny)
    cv = np.zeros(nx * ny)
    for j in range(1, ny - 1):
        for i in range(1, nx - 1):
            ij = i + j * nx
            ia, id_, ig = ij + nx - 1, ij - 1, ij - nx - 1
            ib, ic, if_, ih, ii = ia + 1, ia + 2, ij + 1, ig + 1, ig + 2
            dzdx = ((h[ic] + 2.0 * h[if_] + h[ii]) - (h[ia] + 2.0 * h[id_] + h[ig])) / 8.0 / dx
            dzdy = ((h[ig] + 2.0 * h[ih] + h[ii]) - (h[ia] + 2.0 * h[ib] + h[ic])) / 8.0 / dy
            v = dzdx * dzdx + dzdy * dzdy
            s[ij] = np.arctan(np.sqrt(v)) * con if v > np.finfo(float).tiny else v
            i1, i2, i3, i4, i5, i6, i7, i8, i9 = ia, ib, ic, id_, ij, if_, ig, ih, ii
            a = (h[i1] + h[i3] + h[i4] + h[i6] + h[i7] + h[i9]) / dx / dx / 12.0 - \
                (h[i2] + h[i5] + h[i8]) / dx / dx / 6.0
            b = (h[i1] + h[i2] + h[i3] + h[i7] + h[i8] + h[i9]) / dy / dy / 12.0 - \
                (h[i4] + h[i5] + h[i6]) / dy / dy / 6.0
            c = (h[i3] + h[i7] - h[i1] - h[i9]) / dx / dy / 4.0
            d = (h[i3] + h[i6] + h[i9] - h[i1] - h[i4] - h[i7]) / dx / 6.0
            e = (h[i1] + h[i2] + h[i3] - h[i7] - h[i8] - h[i9]) / dy / 6.0
            v = 1.0 + d * d + e * e
            cv[ij] = (a * (1.0 + e * e) + b * (1.0 + d * d) - c * d * e) / v ** 1.5
    return s, cv


@pytest.mark.parametrize("maker", [lambda: W.plain_d8(23, 19, seed=31, nsteps=3),
                                   lambda: W.mfd(21, 25, seed=32, nsteps=3, bc=1010)])
def test_derived_fields_match_literal(maker):
    """chi, slope, curvature, fluxes and set_all_layers of the oracle against
    plain-Python transliterations of the reference routines."""
    wl = maker()
    wl.apply(O)
    for _ in range(wl.nsteps):
        O.fastscape_execute_step()
    nn = wl.nn
    dx, dy = wl.xl / (wl.nx - 1), wl.yl / (wl.ny - 1)
    buf = np.empty(nn)
    O.fastscape_copy_chi(buf)
    ref = _literal_chi(O.copy_int("stack"), O.copy_int("rec"), O.copy_double("drainage_area"),
                       O.copy_double("length"), dx * dy * 10.0, wl.m / wl.n)
    assert np.array_equal(buf, ref)
    s, cv = _literal_slope_curv(O.copy_double("h"), wl.nx, wl.ny, dx, dy)
    O.fastscape_copy_slope(buf)
    assert np.allclose(buf, s, rtol=1e-14, atol=0)
    O.fastscape_copy_curvature(buf)
    assert np.allclose(buf, cv, rtol=1e-12, atol=1e-12 * np.abs(cv).max())
    # compute_fluxes (FastScape_ctx.f90:843-886)
    erate, u = O.copy_double("erosion_rate"), O.copy_double("u")
    flux = erate.copy()
    if wl.p < -1.5:
        stack, rec = O.copy_int("stack"), O.copy_int("rec")
        for ijk in stack[::-1]:
            flux[ijk] = max(0.0, flux[ijk])
            flux[rec[ijk]] += flux[ijk]
    else:
        mrec, mwrec, mnrec = O.copy_slots("mrec"), O.copy_slots("mwrec"), O.copy_int("mnrec")
        for ijk in O.copy_int("mstack"):
            flux[ijk] = max(0.0, flux[ijk])
            for k in range(mnrec[ijk]):
                flux[mrec[ijk, k]] += flux[ijk] * mwrec[ijk, k]
    bcmask = np.zeros((wl.ny, wl.nx), bool)
    bcmask[0, :] = bcmask[-1, :] = True  # bc 1111 / 1010: bottom and top fixed
    if wl.bc == 1111:
        bcmask[:, 0] = bcmask[:, -1] = True
    surf = wl.xl * wl.yl / (wl.nx - 1) / (wl.ny - 1)
    t, e, b = O.fastscape_get_fluxes()
    assert np.isclose(t, u.sum() * surf, rtol=1e-13)
    assert np.isclose(e, erate.sum() * surf, rtol=1e-13)
    assert np.isclose(b, flux[bcmask.ravel()].sum() * surf, rtol=1e-13)
    # catchment: catch0 of each node's root in the forest before LocalMinima
    catch = O.copy_double("catchment")
    rec_pre = O.copy_int("rec_pre")
    root = np.arange(nn)
    for _ in range(nn):
        nxt = rec_pre[root]
        if np.array_equal(nxt, root):
            break
        root = nxt
    assert np.array_equal(catch, catch[root])  # constant along each pre-LocalMinima tree
    dh = np.linspace(-1.0, 1.0, nn)
    h0, b0 = O.copy_double("h"), O.copy_double("basement")
    O.fastscape_set_all_layers(dh)
    assert np.array_equal(O.copy_double("h"), h0 + dh)
    assert np.array_equal(O.copy_double("basement"), b0 + dh)


def _literal_spl(sfd, h, b, ht_bc, rec, stack, mstack, a, length, mrec, mnrec, mwrec, mlrec, kf, kfsed,
                 m, n, g1, g2, dt, dx, dy):
    """StreamPowerLaw / StreamPowerLawSingleFlowDirection (StreamPowerLaw.f90:3-400)
    with g > 0, statement for statement (0-based ids; lake_sill starts at -1)."""
    nn = h.size
    g = np.full(nn, g1)
    if g2 > 0:
        g[(h - b) > 1.0] = g2
    kfint = kf.copy()
    if kfsed > 0:
        kfint[(h - b) > 1.0] = kfsed
    tol = 1e-4 * (np.max(np.abs(h)) + 1.0)
    err = 2.0 * tol
    ht = h.copy()
    h = h.copy()
    ngs = 0
    lsed = np.zeros(nn)
    lsill = np.full(nn, -1)
    water = np.zeros(nn)
    lwv = np.zeros(nn)
    elev = np.zeros(nn)
    while err > tol and ngs < 99:
        ngs += 1
        hp = h.copy()
        dh = ht - hp
        order = stack[::-1] if sfd else mstack
        for ijk in order:
            if rec[ijk] != ijk:
                dh[ijk] = dh[ijk] - (ht[ijk] - hp[ijk])
                if lsill[ijk] == ijk:
                    lsed[ijk] = 0.0 if dh[ijk] <= 0.0 else dh[ijk]
                dh[ijk] = dh[ijk] + (ht[ijk] - hp[ijk])
                if sfd:
                    dh[rec[ijk]] = dh[rec[ijk]] + dh[ijk]
                else:
                    for k in range(mnrec[ijk]):
                        dh[mrec[ijk, k]] = dh[mrec[ijk, k]] + dh[ijk] * mwrec[ijk, k]
            else:
                lsed[ijk] = dh[ijk]
        for i in range(nn):
            elev[i] = ht[i] if ht_bc[i] else ht[i] + (dh[i] - (ht[i] - hp[i])) * g[i] * dx * dy / a[i]
        omega = 0.875 / n
        for ijk in (stack if sfd else mstack[::-1]):
            ijr = rec[ijk]
            if ijr == ijk:
                water[ijk] = ht[ijk]
                lsill[ijk] = ijk
                lwv[ijk] = 0.0
                continue
            w_rcv = water[ijr]
            if elev[ijk] > w_rcv:
                slots = [(ijr, length[ijk], 1.0)] if sfd else \
                    [(mrec[ijk, k], mlrec[ijk, k], mwrec[ijk, k]) for k in range(mnrec[ijk])]
                if slots:
                    if abs(n - 1.0) < np.finfo(float).tiny:
                        f, df = elev[ijk], 1.0
                        for q, l, w in slots:
                            if sfd or ht[ijk] >= ht[q]:
                                fact = kfint[ijk] * dt * (a[ijk] * w) ** m / l if not sfd else \
                                    kfint[ijk] * dt * a[ijk] ** m / l
                                f = f + fact * h[q]
                                df = df + fact
                        h[ijk] = f / df
                    else:
                        errp, h0 = 2e-3, elev[ijk]
                        while errp > 1e-3:
                            f, df = h[ijk] - h0, 1.0
                            for q, l, w in slots:
                                if ht[ijk] > ht[q]:
                                    fact = kfint[ijk] * dt * a[ijk] ** m / l ** n if sfd else \
                                        kfint[ijk] * dt * (a[ijk] * w) ** m / l ** n
                                    x = max(0.0, h[ijk] - h[q])
                                    f = f + fact * x ** n
                                    df = df + fact * n * x ** (n - 1.0)
                            hn = h[ijk] - f / df
                            errp = abs(hn - h[ijk])
                            h[ijk] = h[ijk] * (1.0 - omega) + hn * omega
                lsill[ijk] = ijk
                lwv[ijk] = 0.0
                if h[ijk] < w_rcv:
                    h[ijk] = w_rcv
            else:
                h[ijk] = elev[ijk]
                lsill[ijk] = lsill[ijr]
                if lsill[ijk] != -1:
                    lwv[lsill[ijk]] = lwv[lsill[ijk]] + (w_rcv - h[ijk])
            water[ijk] = max(w_rcv, h[ijk])
        err = np.sqrt(np.sum((h - hp) ** 2) / nn)
        if np.max(g) < np.finfo(float).tiny:
            err = 0.0
    for ij in range(nn):
        s = lsill[ij]
        if s != -1 and lwv[s] > 0.0:
            h[ij] = h[ij] + max(0.0, min(lsed[s], lwv[s])) / lwv[s] * (water[ij] - h[ij])
    return h, ngs


@pytest.mark.parametrize("nx,ny,bc,p,seed", [(23, 19, 1010, 1.1, 71), (23, 19, 1111, 1.0, 72),
                                             (23, 19, 101, -1.0, 73), (23, 19, 1000, 0.0, 74),
                                             (3, 4, 1000, 1.1, 75), (4, 3, 101, -1.0, 76)])
def test_mfd_routing_matches_literal(nx, ny, bc, p, seed):
    """The oracle's multiple-flow routing (find_mult_rec: fill, receivers with
    their clamp duplicates, weights and the p < 0 single-precision exponent,
    lengths, the LIFO mstack) and its drainage area against a literal
    transliteration, bit for bit.  With no uplift the routing sees init_h's h;
    rec and stack are the oracle's single-flow result after LocalMinima, which
    test_routing_matches_literal pins separately."""
    wl = W.mfd(nx, ny, seed=seed, nsteps=1, p=p, bc=bc)
    wl.u = np.zeros(wl.nn)
    wl.apply(O)
    O.fastscape_execute_step()
    nn = wl.nn
    dx, dy = wl.xl / (nx - 1), wl.yl / (ny - 1)
    _, bounds = FL.set_bc(nx, ny, wl.bc)
    rec0 = [0] + [r + 1 for r in O.copy_int("rec").tolist()]
    stack0 = [0] + [s + 1 for s in O.copy_int("stack").tolist()]
    rec, nrec, wrec, lrec, mstack, water, _ = FL.find_mult_rec(
        [0.0] + wl.h0.tolist(), rec0, stack0, nx, ny, dx, dy, p, [0.0] + [p] * nn, bounds)
    assert nrec[1:] == O.copy_int("mnrec").tolist()
    assert nn < 20 or sum(nrec) > nn  # on the larger grids many nodes have several receivers
    mrec, mw, ml = O.copy_slots("mrec"), O.copy_slots("mwrec"), O.copy_slots("mlrec")
    for ij in range(1, nn + 1):
        k = nrec[ij]
        assert [r - 1 for r in rec[ij][1:k + 1]] == mrec[ij - 1, :k].tolist()
        assert wrec[ij][1:k + 1] == mw[ij - 1, :k].tolist()
        assert lrec[ij][1:k + 1] == ml[ij - 1, :k].tolist()
    assert [s - 1 for s in mstack[1:]] == O.copy_int("mstack").tolist()
    assert water[1:] == O.copy_double("hwater").tolist()
    a = FL.flow_accumulation_mfd(mstack, rec, nrec, wrec, [0.0] + [1.0] * nn, nn, dx, dy)
    assert a[1:] == O.copy_double("drainage_area").tolist()


@pytest.mark.parametrize("sfd,n,kfsed,g2", [(True, 1.0, -1.0, 0.0), (True, 1.5, -1.0, 0.0),
                                             (False, 1.0, -1.0, 0.0), (False, 1.5, -1.0, 0.0),
                                             (True, 1.0, 3e-4, 0.6), (False, 1.5, 5e-5, 0.6)])
def test_sediment_spl_matches_literal(sfd, n, kfsed, g2):
    """The oracle's g > 0 stream power law against a literal transliteration:
    with no uplift and no diffusion a step's change of h is the SPL alone.
    With kfsed and g2 set, nodes with more than 1 m of sediment above the
    basement take them instead of kf and g1 (StreamPowerLaw.f90:236-243)."""
    wl = W.plain_d8(19, 17, seed=51) if sfd else W.mfd(19, 17, seed=52, p=1.1, bc=1111)
    wl.n, wl.g1, wl.g2, wl.kfsed = n, 1.2, g2, kfsed
    wl.kf = np.full(wl.nn, (1e-4 if n == 1.0 else 2e-3) if sfd else 2e-5)
    wl.u = np.zeros(wl.nn)
    wl.kd = np.zeros(wl.nn)
    wl.apply(O)
    if kfsed > 0.0:  # sediment thicker than 1 m on half of the nodes
        rng = np.random.default_rng(57)
        O.fastscape_set_basement(wl.h0 - np.where(rng.random(wl.nn) < 0.5, 3.0, 0.0))
    for _ in range(2):
        O.fastscape_execute_step()
    h0, b0 = O.copy_double("h"), O.copy_double("basement")
    O.fastscape_execute_step()
    bc = np.zeros((wl.ny, wl.nx), bool)
    bc[0, :] = bc[-1, :] = bc[:, 0] = bc[:, -1] = True
    dx, dy = wl.xl / (wl.nx - 1), wl.yl / (wl.ny - 1)
    h_lit, ngs = _literal_spl(sfd, h0, b0, bc.ravel(), O.copy_int("rec"), O.copy_int("stack"),
                              O.copy_int("mstack"), O.copy_double("drainage_area"),
                              O.copy_double("length"), O.copy_slots("mrec"), O.copy_int("mnrec"),
                              O.copy_slots("mwrec"), O.copy_slots("mlrec"), wl.kf, wl.kfsed, wl.m, n,
                              wl.g1, wl.g2, wl.dt, dx, dy)
    assert ngs == O.get_ngs() and ngs > 1
    assert np.max(np.abs(O.copy_double("h") - h_lit)) <= 1e-12 * (np.abs(h_lit).max() + 1.0)


@pytest.mark.parametrize("sfd,n", [(False, 1.5), (False, 1.0), (True, 1.5), (True, 1.0)])
def test_spl_g0_matches_literal(sfd, n):
    """The oracle's stream power law as the benchmark runs it (g = 0: one
    Gauss-Seidel pass; multiple flow with Newton at n = 1.5 first) against the
    literal transliteration; no uplift and no diffusion, so a step's change of
    h is the SPL alone."""
    wl = W.plain_d8(19, 17, seed=53) if sfd else W.mfd(19, 17, seed=54, p=1.1, bc=1010)
    wl.n, wl.g1, wl.g2 = n, 0.0, 0.0
    wl.kf = np.full(wl.nn, (1e-4 if n == 1.0 else 2e-3) if sfd else 2e-5)
    wl.u = np.zeros(wl.nn)
    wl.kd = np.zeros(wl.nn)
    wl.apply(O)
    for _ in range(2):
        O.fastscape_execute_step()
    h0, b0 = O.copy_double("h"), O.copy_double("basement")
    O.fastscape_execute_step()
    _, (i1, i2, j1, j2, xc, yc) = FL.set_bc(wl.nx, wl.ny, wl.bc)
    ii, jj = np.meshgrid(np.arange(1, wl.nx + 1), np.arange(1, wl.ny + 1))
    fixed = ((ii < i1) | (ii > i2) | (jj < j1) | (jj > j2)).ravel()
    dx, dy = wl.xl / (wl.nx - 1), wl.yl / (wl.ny - 1)
    h_lit, ngs = _literal_spl(sfd, h0, b0, fixed, O.copy_int("rec"), O.copy_int("stack"),
                              O.copy_int("mstack"), O.copy_double("drainage_area"),
                              O.copy_double("length"), O.copy_slots("mrec"), O.copy_int("mnrec"),
                              O.copy_slots("mwrec"), O.copy_slots("mlrec"), wl.kf, wl.kfsed, wl.m, n,
                              wl.g1, wl.g2, wl.dt, dx, dy)
    assert ngs == 1
    dh = np.abs(O.copy_double("h") - h0)
    assert dh.max() > 0.0  # the step eroded something
    assert np.max(np.abs(O.copy_double("h") - h_lit)) <= 1e-12 * (np.abs(h_lit).max() + 1.0)


def _tridag(a, b, c, r):
    """tridag (Diffusion.f90:164-202), 0-based."""
    n = len(b)
    u, gam = np.zeros(n), np.zeros(n)
    bet = b[0]
    u[0] = r[0] / bet
    for j in range(1, n):
        gam[j] = c[j - 1] / bet
        bet = b[j] - a[j] * gam[j]
        u[j] = (r[j] - a[j] * u[j - 1]) / bet
    for j in range(n - 2, -1, -1):
        u[j] = u[j] - gam[j + 1] * u[j + 1]
    return u


def _literal_diffusion(h, b, kd, kdsed, nx, ny, dx, dy, dt, jbc):
    """Diffusion (Diffusion.f90:1-160), statement for statement on 1-based
    (i, j) arrays; returns h, b, and the etot and erate increments.  The
    bottom-boundary branch reads kdint(i, j) with j = ny, the value the
    preceding loop leaves (Diffusion.f90:114)."""
    cbc = "****" if (jbc > 9999 or jbc < -999) else "%4d" % jbc
    z = np.zeros((nx + 2, ny + 2))
    kdi = np.zeros((nx + 2, ny + 2))
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            ij = (j - 1) * nx + i - 1
            z[i, j] = h[ij]
            kdi[i, j] = kd[ij]
            if kdsed > 0.0 and (h[ij] - b[ij]) > 1.0e-6:
                kdi[i, j] = kdsed
    zp = z.copy()
    hdt = dt / 2.0
    fx = lambda a, c: (a + c) / 2.0 * hdt / (dx * dx)  # noqa: E731
    fy = lambda a, c: (a + c) / 2.0 * hdt / (dy * dy)  # noqa: E731
    for j in range(2, ny):
        diag, sup, inf, f = np.zeros(nx + 1), np.zeros(nx + 1), np.zeros(nx + 1), np.zeros(nx + 1)
        for i in range(2, nx):
            fxp, fxm = fx(kdi[i + 1, j], kdi[i, j]), fx(kdi[i - 1, j], kdi[i, j])
            fyp, fym = fy(kdi[i, j + 1], kdi[i, j]), fy(kdi[i, j - 1], kdi[i, j])
            diag[i] = 1.0 + fxp + fxm
            sup[i] = -fxp
            inf[i] = -fxm
            f[i] = zp[i, j] + fyp * zp[i, j + 1] - (fyp + fym) * zp[i, j] + fym * zp[i, j - 1]
        if cbc[3] == "1":
            diag[1], sup[1], f[1] = 1.0, 0.0, zp[1, j]
        else:
            fxp, fyp, fym = fx(kdi[2, j], kdi[1, j]), fy(kdi[1, j + 1], kdi[1, j]), fy(kdi[1, j - 1], kdi[1, j])
            diag[1], sup[1] = 1.0 + fxp, -fxp
            f[1] = zp[1, j] + fyp * zp[1, j + 1] - (fyp + fym) * zp[1, j] + fym * zp[1, j - 1]
        if cbc[1] == "1":
            diag[nx], inf[nx], f[nx] = 1.0, 0.0, zp[nx, j]
        else:
            fxm = fx(kdi[nx - 1, j], kdi[nx, j])
            fyp, fym = fy(kdi[nx, j + 1], kdi[nx, j]), fy(kdi[nx, j - 1], kdi[nx, j])
            diag[nx], inf[nx] = 1.0 + fxm, -fxm
            f[nx] = zp[nx, j] + fyp * zp[nx, j + 1] - (fyp + fym) * zp[nx, j] + fym * zp[nx, j - 1]
        z[1:nx + 1, j] = _tridag(inf[1:], diag[1:], sup[1:], f[1:])
    for i in range(2, nx):
        diag, sup, inf, f = np.zeros(ny + 1), np.zeros(ny + 1), np.zeros(ny + 1), np.zeros(ny + 1)
        for j in range(2, ny):
            fxp, fxm = fx(kdi[i + 1, j], kdi[i, j]), fx(kdi[i - 1, j], kdi[i, j])
            fyp, fym = fy(kdi[i, j + 1], kdi[i, j]), fy(kdi[i, j - 1], kdi[i, j])
            diag[j] = 1.0 + fyp + fym
            sup[j] = -fyp
            inf[j] = -fym
            f[j] = z[i, j] + fxp * z[i + 1, j] - (fxp + fxm) * z[i, j] + fxm * z[i - 1, j]
        jq = ny  # the loop variable after `do j=2,ny-1`
        if cbc[0] == "1":
            diag[1], sup[1], f[1] = 1.0, 0.0, z[i, 1]
        else:
            fxp, fxm = fx(kdi[i + 1, 1], kdi[i, jq]), fx(kdi[i - 1, 1], kdi[i, 1])
            fyp = fy(kdi[i, 2], kdi[i, 1])
            diag[1], sup[1] = 1.0 + fyp, -fyp
            f[1] = z[i, 1] + fxp * z[i + 1, 1] - (fxp + fxm) * z[i, 1] + fxm * z[i - 1, 1]
        if cbc[2] == "1":
            diag[ny], inf[ny], f[ny] = 1.0, 0.0, z[i, ny]
        else:
            fxp, fxm = fx(kdi[i + 1, ny], kdi[i, ny]), fx(kdi[i - 1, ny], kdi[i, ny])
            fym = fy(kdi[i, ny - 1], kdi[i, ny])
            diag[ny], inf[ny] = 1.0 + fym, -fym
            f[ny] = z[i, ny] + fxp * z[i + 1, ny] - (fxp + fxm) * z[i, ny] + fxm * z[i - 1, ny]
        zp[i, 1:ny + 1] = _tridag(inf[1:], diag[1:], sup[1:], f[1:])
    hn = zp[1:nx + 1, 1:ny + 1].T.ravel().copy()
    return hn, np.minimum(hn, b), h - hn, (h - hn) / dt


@pytest.mark.parametrize("nx,ny,bc,kdsed,seed", [(17, 13, 1111, -1.0, 81), (17, 13, 1010, 0.05, 82),
                                                 (17, 13, 101, -1.0, 83), (17, 13, 1000, 0.05, 84),
                                                 (3, 3, 101, -1.0, 85), (4, 5, 1000, 0.05, 86)])
def test_diffusion_matches_literal(nx, ny, bc, kdsed, seed):
    """The oracle's ADI diffusion against a literal transliteration, bit for
    bit: no uplift and kf = 0 (the stream power law then leaves h as it is),
    so a step's change of h, b, etot and erate is the diffusion alone; a
    spatially varying kd, and kdsed on nodes with sediment above the basement."""
    wl = W.plain_d8(nx, ny, seed=seed)
    rng = np.random.default_rng(seed)
    wl.bc = bc
    wl.kdsed = kdsed
    wl.kf = np.zeros(wl.nn)
    wl.u = np.zeros(wl.nn)
    wl.kd = 1.0e2 * (0.5 + rng.random(wl.nn))
    wl.apply(O)
    b = wl.h0 - np.where(rng.random(wl.nn) < 0.5, 2.0, 0.0)
    O.fastscape_set_basement(b)
    O.fastscape_execute_step()
    dx, dy = wl.xl / (wl.nx - 1), wl.yl / (wl.ny - 1)
    h, bl, de, dr = _literal_diffusion(wl.h0, b, wl.kd, kdsed, wl.nx, wl.ny, dx, dy, wl.dt, bc)
    assert nx * ny < 12 or np.max(np.abs(h - wl.h0)) > 0.0  # the step diffused something
    np.testing.assert_array_equal(O.copy_double("h"), h)
    np.testing.assert_array_equal(O.copy_double("basement"), bl)
    np.testing.assert_array_equal(O.copy_double("total_erosion"), de)
    np.testing.assert_array_equal(O.copy_double("erosion_rate"), dr)


def _literal_advect(h, b, etot, vx, vy, nx, ny, dx, dy, dt):
    """Advect (Advect.f90:1-103) on (ny, nx) arrays."""
    h, b, etot = h.reshape(ny, nx).copy(), b.reshape(ny, nx).copy(), etot.reshape(ny, nx).copy()
    vx, vy = vx.reshape(ny, nx), vy.reshape(ny, nx)

    def coefs(v, d):
        n = v.size
        diag, sup, inf = np.ones(n), np.zeros(n), np.zeros(n)
        for i in range(n):
            if v[i] > 0.0:
                diag[i] = 1.0 + v[i] * dt / d
                inf[i] = -(v[i] * dt / d)
            elif v[i] < 0.0:
                diag[i] = 1.0 - v[i] * dt / d
                sup[i] = v[i] * dt / d
        sup[0], diag[0], diag[-1], inf[-1] = 0.0, 1.0, 1.0, 0.0
        return inf, diag, sup

    for j in range(ny):
        inf, diag, sup = coefs(vx[j, :], dx)
        for f in (h, b, etot):
            f[j, :] = _tridag(inf, diag, sup, f[j, :])
    for i in range(nx):
        inf, diag, sup = coefs(vy[:, i], dy)
        for f in (h, b, etot):
            f[:, i] = _tridag(inf, diag, sup, f[:, i])
    return h.ravel(), np.minimum(b, h).ravel(), etot.ravel()


def velocity_field(nx, ny, seed):
    rng = np.random.default_rng(seed)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    vx = 0.02 * np.sin(2 * np.pi * j / ny) + 0.005 * rng.standard_normal((ny, nx))
    vy = 0.015 * np.cos(2 * np.pi * i / nx) + 0.005 * rng.standard_normal((ny, nx))
    vx[:, nx // 3] = 0.0  # zero velocities take the diag = 1 branch
    return vx.ravel(), vy.ravel()


def test_advect_matches_literal():
    """The oracle's Advect against a literal transliteration (no uplift, no
    erosion, no diffusion: a step is the advection alone)."""
    wl = W.plain_d8(23, 19, seed=61)
    wl.kf = np.zeros(wl.nn)
    wl.kd = np.zeros(wl.nn)
    wl.u = np.zeros(wl.nn)
    wl.apply(O)
    vx, vy = velocity_field(wl.nx, wl.ny, 7)
    O.fastscape_set_v(vx, vy)
    h0, b0, e0 = O.copy_double("h"), O.copy_double("basement"), O.copy_double("total_erosion")
    O.fastscape_execute_step()
    dx, dy = wl.xl / (wl.nx - 1), wl.yl / (wl.ny - 1)
    h, b, e = _literal_advect(h0, b0, e0, vx, vy, wl.nx, wl.ny, dx, dy, wl.dt)
    assert np.array_equal(O.copy_double("h"), h)
    assert np.array_equal(O.copy_double("basement"), b)
    assert np.array_equal(O.copy_double("total_erosion"), e)


def literal_vtk_bytes(nx, ny, xl, yl, step, z, scal_name, scal, f, vex):
    """The bytes of one Make_VTK file (FastScape_ctx.f90:692-777), gfortran
    with -fconvert=big-endian (CMakeLists.txt:49)."""
    import struct
    nn = nx * ny
    dx, dy = xl / (nx - 1), yl / (ny - 1)
    nnc = "%12d" % nn
    out = bytearray(("# vtk DataFile Version 3.0\nFastScape\nBINARY\nDATASET STRUCTURED_GRID\n"
                     "DIMENSIONS %6d %6d 1\nPOINTS%s float\n" % (nx, ny, nnc)).encode())
    pts = np.empty((nn, 3), dtype=np.float64)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    pts[:, 0] = dx * ii.ravel()
    pts[:, 1] = dy * jj.ravel()
    pts[:, 2] = z * abs(vex)
    out += pts.astype(">f4").tobytes()
    out += ("POINT_DATA%s\n" % nnc).encode()
    out += ("SCALARS %s float 1\nLOOKUP_TABLE default\n" % scal_name).encode()
    out += np.asarray(scal, dtype=np.float64).astype(">f4").tobytes()
    if f is not None:
        out += b"SCALARS HHHHH float 1\nLOOKUP_TABLE default\n"
        out += np.asarray(f, dtype=np.float64).astype(">f4").tobytes()
    assert struct.calcsize(">f") == 4
    return bytes(out)


def test_vtk_matches_literal(tmp_path):
    wl = W.plain_d8(13, 11, seed=81)
    wl.apply(O)
    O.fastscape_execute_step()
    f = np.random.default_rng(3).standard_normal(wl.nn) * 1e3
    O.fastscape_vtk(f, -2.0, str(tmp_path))
    h, b = O.copy_double("h"), O.copy_double("basement")
    args = (wl.nx, wl.ny, wl.xl, wl.yl, 1)
    assert (tmp_path / "Topography0000001.vtk").read_bytes() == literal_vtk_bytes(*args, h, "H", h, f, -2.0)
    assert (tmp_path / "Basement0000001.vtk").read_bytes() == literal_vtk_bytes(*args, b, "B", b, f, -2.0)
    zero = np.zeros(wl.nn)
    assert (tmp_path / "SeaLevel0000001.vtk").read_bytes() == literal_vtk_bytes(*args, zero, "SL", zero, None, -2.0)
