"""Literal pure-Python transliteration of the reference's single-flow routing and
depression re-routing, used only by the tests as a second, independent
restatement that the C++ oracle is checked against on small grids.

Arrays are 1-based (index 0 unused) and loops keep the Fortran control flow,
including the goto structure of the Numerical Recipes index sort.
Reference file:line for each routine is given in its docstring.
"""
from __future__ import annotations

import math
import struct
import sys

TINY = sys.float_info.min


def set_bc(nx, ny, jbc):
    """SetBC -- src/FastScape_ctx.f90:565-593."""
    cbc = "****" if (jbc > 9999 or jbc < -999) else "%4d" % jbc
    nn = nx * ny
    bc = [False] * (nn + 1)
    i1, i2, j1, j2 = 1, nx, 1, ny
    if cbc[3] == "1":
        i1 = 2
    if cbc[1] == "1":
        i2 = nx - 1
    if cbc[0] == "1":
        j1 = 2
    if cbc[2] == "1":
        j2 = ny - 1
    if cbc[3] == "1":
        for ij in range(1, nn + 1, nx):
            bc[ij] = True
    if cbc[1] == "1":
        for ij in range(nx, nn + 1, nx):
            bc[ij] = True
    if cbc[0] == "1":
        for ij in range(1, nx + 1):
            bc[ij] = True
    if cbc[2] == "1":
        for ij in range(nx * (ny - 1) + 1, nn + 1):
            bc[ij] = True
    xc = cbc[3] != "1" and cbc[1] != "1"
    yc = cbc[0] != "1" and cbc[2] != "1"
    return bc, (i1, i2, j1, j2, xc, yc)


def find_receiver(h, nx, ny, dx, dy, bounds):
    """find_receiver -- src/FlowRouting.f90:302-362."""
    i1, i2, j1, j2, xc, yc = bounds
    nn = nx * ny
    rec = list(range(nn + 1))
    length = [0.0] * (nn + 1)
    for j in range(j1, j2 + 1):
        for i in range(i1, i2 + 1):
            ij = i + (j - 1) * nx
            smax = TINY
            for jj in (-1, 0, 1):
                for ii in (-1, 0, 1):
                    iii = i + ii
                    if iii < 1 and xc:
                        iii += nx
                    iii = max(iii, 1)
                    if iii > nx and xc:
                        iii -= nx
                    iii = min(iii, nx)
                    jjj = j + jj
                    if jjj < 1 and yc:
                        jjj += ny
                    jjj = max(jjj, 1)
                    if jjj > ny and yc:
                        jjj -= ny
                    jjj = min(jjj, ny)
                    ijk = iii + (jjj - 1) * nx
                    if ijk != ij:
                        ax, ay = dx * ii, dy * jj
                        l = math.sqrt(ax * ax + ay * ay)
                        slope = (h[ij] - h[ijk]) / l
                        if slope > smax:
                            smax = slope
                            rec[ij] = ijk
                            length[ij] = l
    return rec, length


def find_donor(rec, nn):
    """find_donor -- src/FlowRouting.f90:366-389."""
    ndon = [0] * (nn + 1)
    don = [[0] * 9 for _ in range(nn + 1)]
    for ij in range(1, nn + 1):
        if rec[ij] != ij:
            ijk = rec[ij]
            ndon[ijk] += 1
            don[ijk][ndon[ijk]] = ij
    return ndon, don


def find_stack(rec, don, ndon, nn):
    """find_stack + find_stack_recursively -- src/FlowRouting.f90:393-443."""
    stack = [0] * (nn + 1)
    nstack = [0]
    sys.setrecursionlimit(max(10000, 4 * nn))

    def rec_(ij):
        for k in range(1, ndon[ij] + 1):
            ijk = don[ij][k]
            nstack[0] += 1
            stack[nstack[0]] = ijk
            rec_(ijk)

    for ij in range(1, nn + 1):
        if rec[ij] == ij:
            nstack[0] += 1
            stack[nstack[0]] = ij
            rec_(ij)
    return stack


def compute_basins(stack, rec, n):
    """compute_basins -- src/LocalMinima.f90:136-169."""
    basins = [0] * (n + 1)
    outlets = [0] * (n + 1)
    ib = 0
    for i in range(1, n + 1):
        s = stack[i]
        if rec[s] == s:
            ib += 1
            outlets[ib] = s
        basins[s] = ib
    return basins, outlets, ib


def connect_basins(nbasins, basins, outlets, rec, stack, active, h, nx, ny):
    """connect_basins -- src/LocalMinima.f90:173-329."""
    n = nx * ny
    ii = [-1, 1, 0, 0, -1, 1, -1, 1]
    jj = [0, 0, -1, 1, -1, -1, 1, 1]
    cb, cn, cw = [], [], []
    basin0 = -1
    ibasin = 1
    conn_pos = [-1] * (nbasins + 1)
    used = []
    act = False
    for iis in range(1, n + 1):
        s = stack[iis]
        if rec[s] == s:
            ibasin = basins[s]
            act = active[s]
            for u in used:
                conn_pos[u] = -1
            used = []
            if not act:
                if basin0 == -1:
                    basin0 = ibasin
                else:
                    cb.append([basin0, ibasin])
                    cn.append([-1, -1])
                    cw.append(-1.0e10)
        if act:
            i = (s - 1) % nx + 1
            j = (s - 1) // nx + 1
            for k in range(8):
                ki, kj = i + ii[k], j + jj[k]
                if ki < 1 or ki > nx or kj < 1 or kj > ny:
                    continue
                nb = (kj - 1) * nx + ki
                nbb = basins[nb]
                if ibasin >= nbb and active[outlets[nbb]]:
                    continue
                w = max(h[s], h[nb])
                ci = conn_pos[nbb]
                if ci == -1:
                    cb.append([ibasin, nbb])
                    cn.append([s, nb])
                    cw.append(w)
                    conn_pos[nbb] = len(cw)
                    used.append(nbb)
                elif w < cw[ci - 1]:
                    cn[ci - 1] = [s, nb]
                    cw[ci - 1] = w
    return basin0, cb, cn, cw


def indexx(arr):
    """loc_min_3_indexx -- src/LocalMinima.f90:947-1046 (labels 1-5 kept).

    ``arr`` is 0-based; the returned permutation is 1-based like indx(1:n)."""
    n = len(arr)
    A = [0.0] + list(arr)
    M, NSTACK = 7, 50
    indx = list(range(n + 1))
    istack = [0] * (NSTACK + 1)
    jstack, l, ir = 0, 1, n
    while True:  # label 1
        if ir - l < M:
            for j in range(l + 1, ir + 1):
                indxt = indx[j]
                a = A[indxt]
                i = j - 1
                while i >= 1:
                    if A[indx[i]] <= a:
                        break  # goto 2
                    indx[i + 1] = indx[i]
                    i -= 1
                else:
                    i = 0
                indx[i + 1] = indxt  # label 2
            if jstack == 0:
                return indx[1:]
            ir = istack[jstack]
            l = istack[jstack - 1]
            jstack -= 2
        else:
            k = (l + ir) // 2
            indx[k], indx[l + 1] = indx[l + 1], indx[k]
            if A[indx[l + 1]] > A[indx[ir]]:
                indx[l + 1], indx[ir] = indx[ir], indx[l + 1]
            if A[indx[l]] > A[indx[ir]]:
                indx[l], indx[ir] = indx[ir], indx[l]
            if A[indx[l + 1]] > A[indx[l]]:
                indx[l + 1], indx[l] = indx[l], indx[l + 1]
            i, j = l + 1, ir
            indxt = indx[l]
            a = A[indxt]
            while True:
                i += 1  # label 3
                while A[indx[i]] < a:
                    i += 1
                j -= 1  # label 4
                while A[indx[j]] > a:
                    j -= 1
                if j < i:
                    break  # goto 5
                indx[i], indx[j] = indx[j], indx[i]
            indx[l] = indx[j]  # label 5
            indx[j] = indxt
            jstack += 2
            if jstack > NSTACK:
                raise RuntimeError("NSTACK too small in loc_min_3_indexx")
            if ir - i + 1 >= j - l:
                istack[jstack] = ir
                istack[jstack - 1] = i
                ir = j - 1
            else:
                istack[jstack] = j - 1
                istack[jstack - 1] = l
                l = i


def union_find(x, parent):
    """UnionFind -- src/LocalMinima.f90:815-832."""
    xp, xc = x, -1000
    while xc != xp:
        xc = xp
        xp = parent[xc]
    parent[x] = xc
    return xc


def mst_kruskal(cw, cb, nbasins):
    """mst_kruskal + DoUnion -- src/LocalMinima.f90:333-385, 783-811."""
    sort_id = indexx(cw)
    parent = list(range(nbasins + 1))
    rank = [0] * (nbasins + 1)
    tree = []
    for eid in sort_id:
        b0, b1 = cb[eid - 1]
        f0, f1 = union_find(b0, parent), union_find(b1, parent)
        if f0 != f1:
            tree.append(eid)
            xr, yr = union_find(b0, parent), union_find(b1, parent)
            if xr != yr:
                if rank[xr] < rank[yr]:
                    parent[xr] = yr
                else:
                    parent[yr] = xr
                    if rank[xr] == rank[yr]:
                        rank[xr] += 1
    return sort_id, tree


def order_tree(cb, cn, nbasins, root, tree):
    """order_tree -- src/LocalMinima.f90:389-533 (continuous_flow=.false.)."""
    size = [0] * (nbasins + 1)
    ptr = [0] * (nbasins + 1)
    for i in tree:
        size[cb[i - 1][0]] += 1
        size[cb[i - 1][1]] += 1
    ptr[1] = 1
    for i in range(2, nbasins + 1):
        ptr[i] = ptr[i - 1] + size[i - 1]
        size[i - 1] = 0
    adj = [0] * (ptr[nbasins] + size[nbasins] + 1)
    size[nbasins] = 0
    for i in tree:
        n1, n2 = cb[i - 1]
        adj[ptr[n1] + size[n1]] = i
        adj[ptr[n2] + size[n2]] = i
        size[n1] += 1
        size[n2] += 1
    st = [(root, root)]
    while st:
        node, parent = st.pop()
        for i in range(ptr[node], ptr[node] + size[node]):
            e = adj[i] - 1
            if cb[e][0] == parent and node != parent:
                continue
            if node != cb[e][0]:
                cb[e] = [cb[e][1], cb[e][0]]
                cn[e] = [cn[e][1], cn[e][0]]
            st.append((cb[e][1], node))


def correct_receivers_v2(rec, length, outlets, cb, cn, tree, nx, dx, dy):
    """correct_receivers_v2 -- src/LocalMinima.f90:601-662."""
    for i in tree:
        node_to, node_from = cn[i - 1]
        if node_from == -1:
            continue
        outlet_from = outlets[cb[i - 1][1]]
        nxt = rec[node_from]
        cur = node_from
        prev = length[node_from]
        rec[node_from] = node_to
        ddx = dx * float(((node_from - 1) % nx) - ((node_to - 1) % nx))
        ddy = dy * float(((node_from - 1) // nx) - ((node_to - 1) // nx))
        length[node_from] = math.sqrt(ddx * ddx + ddy * ddy)
        while cur != outlet_from:
            r = rec[nxt]
            rec[nxt] = cur
            tmp = prev
            prev = length[nxt]
            length[nxt] = tmp
            cur = nxt
            nxt = r


def routing_sfd(h0, nx, ny, dx, dy, jbc):
    """FlowRoutingSingleFlowDirection up to the lake fill (FlowRouting.f90:43-89)
    with LocalMinima (LocalMinima.f90:1-132).  ``h0`` is 0-based."""
    nn = nx * ny
    h = [0.0] + list(h0)
    bc, bounds = set_bc(nx, ny, jbc)
    rec, length = find_receiver(h, nx, ny, dx, dy, bounds)
    ndon, don = find_donor(rec, nn)
    stack = find_stack(rec, don, ndon, nn)
    out = {"rec_pre": rec[1:], "stack_pre": stack[1:]}
    basins, outlets, nb = compute_basins(stack, rec, nn)
    active = [not b for b in bc]
    basin0, cb, cn, cw = connect_basins(nb, basins, outlets, rec, stack, active, h, nx, ny)
    sort_id, tree = mst_kruskal(cw, cb, nb)
    out.update(basins=basins[1:], nbasins=nb, basin0=basin0, cb=[list(x) for x in cb],
               cn=[list(x) for x in cn], cw=list(cw), sort_id=sort_id, tree=list(tree))
    order_tree(cb, cn, nb, basin0, tree)
    out.update(ocb=cb, ocn=cn)
    correct_receivers_v2(rec, length, outlets, cb, cn, tree, nx, dx, dy)
    ndon, don = find_donor(rec, nn)
    stack = find_stack(rec, don, ndon, nn)
    out.update(rec=rec[1:], length=length[1:], stack=stack[1:], ndon=ndon[1:],
               don=[don[k][1:ndon[k] + 1] for k in range(1, nn + 1)], rec_1b=rec, stack_1b=stack)
    return out


def find_mult_rec(h, rec0, stack0, nx, ny, dx, dy, p, p_mfd_exp, bounds):
    """find_mult_rec -- src/FlowRouting.f90:147-298.  ``h``, ``rec0``, ``stack0``
    and ``p_mfd_exp`` are 1-based; returns (rec, nrec, wrec, lrec, stack,
    water, p_mfd_exp), 1-based, with rec/wrec/lrec as lists of 8-slot lists."""
    i1, i2, j1, j2, xc, yc = bounds
    nn = nx * ny
    h0 = list(h)
    deltah = 1.0e-8
    for i in range(1, nn + 1):  # :187-196
        ijk = stack0[i]
        ijr = rec0[ijk]
        if ijr != 0:
            if h0[ijr] > h0[ijk]:
                h0[ijk] = h0[ijr] + deltah
    water = list(h0)
    nrec = [0] * (nn + 1)
    rec = [[0] * 9 for _ in range(nn + 1)]
    wrec = [[0.0] * 9 for _ in range(nn + 1)]
    lrec = [[0.0] * 9 for _ in range(nn + 1)]
    for j in range(j1, j2 + 1):  # :204-230
        for i in range(i1, i2 + 1):
            ij = (j - 1) * nx + i
            for jj in (-1, 0, 1):
                jjj = j + jj
                if jjj < 1 and yc:
                    jjj = jjj + ny
                jjj = max(jjj, 1)
                if jjj > ny and yc:
                    jjj = jjj - ny
                jjj = min(jjj, ny)
                for ii in (-1, 0, 1):
                    iii = i + ii
                    if iii < 1 and xc:
                        iii = iii + nx
                    iii = max(iii, 1)
                    if iii > nx and xc:
                        iii = iii - nx
                    iii = min(iii, nx)
                    ijk = (jjj - 1) * nx + iii
                    if h0[ij] > h0[ijk]:
                        nrec[ij] += 1
                        k = nrec[ij]
                        rec[ij][k] = ijk
                        lrec[ij][k] = math.sqrt((ii * dx) * (ii * dx) + (jj * dy) * (jj * dy))
                        wrec[ij][k] = (h0[ij] - h0[ijk]) / lrec[ij][k]
    pexp = list(p_mfd_exp)
    f32 = lambda x: struct.unpack("f", struct.pack("f", x))[0]  # noqa: E731  Fortran real()
    for ij in range(1, nn + 1):  # :232-243
        if p < 0.0:
            slope = 0.0
            if nrec[ij] != 0:
                s = 0.0
                for k in range(1, nrec[ij] + 1):
                    s = s + wrec[ij][k]
                slope = f32(s / nrec[ij])
            pexp[ij] = f32(0.5) + f32(0.6) * slope
        for k in range(1, nrec[ij] + 1):
            wrec[ij][k] = wrec[ij][k] ** pexp[ij]
        sumweight = 0.0
        for k in range(1, nrec[ij] + 1):
            sumweight = sumweight + wrec[ij][k]
        for k in range(1, nrec[ij] + 1):
            wrec[ij][k] = wrec[ij][k] / sumweight
    ndon = [0] * (nn + 1)  # :247-255
    for ij in range(1, nn + 1):
        for k in range(1, nrec[ij] + 1):
            ndon[rec[ij][k]] += 1
    stack = [0] * (nn + 1)  # :259-292, LIFO parse stack
    vis = [0] * (nn + 1)
    parse = []
    nstack = 0
    for ij in range(1, nn + 1):
        if ndon[ij] == 0:
            parse.append(ij)
        while parse:
            ijn = parse.pop()
            nstack += 1
            stack[nstack] = ijn
            for k in range(1, nrec[ijn] + 1):
                ijr = rec[ijn][k]
                vis[ijr] += 1
                if vis[ijr] == ndon[ijr]:
                    parse.append(ijr)
    if nstack != nn:
        raise RuntimeError("error in stack")
    return rec, nrec, wrec, lrec, stack, water, pexp


def flow_accumulation_mfd(mstack, mrec, mnrec, mwrec, precip, nn, dx, dy):
    """FlowAccumulation -- src/FlowRouting.f90:97-119 (1-based)."""
    a = [0.0] + [dx * dy * precip[ij] for ij in range(1, nn + 1)]
    for ij in range(1, nn + 1):
        ijk = mstack[ij]
        for k in range(1, mnrec[ijk] + 1):
            a[mrec[ijk][k]] = a[mrec[ijk][k]] + a[ijk] * mwrec[ijk][k]
    return a


def lake_fill_sfd(h, rec, stack, nn):
    """hwater of FlowRoutingSingleFlowDirection -- src/FlowRouting.f90:73-89 (1-based)."""
    hwater = list(h)
    deltah = 1.0e-8
    for i in range(1, nn + 1):
        ijk = stack[i]
        ijr = rec[ijk]
        if ijr != 0:
            if hwater[ijr] > hwater[ijk]:
                hwater[ijk] = hwater[ijr] + deltah
    return hwater


def flow_accumulation_sfd(stack, rec, precip, nn, dx, dy):
    """FlowAccumulationSingleFlowDirection -- src/FlowRouting.f90:123-143 (1-based)."""
    a = [0.0] + [dx * dy * precip[ij] for ij in range(1, nn + 1)]
    for ij in range(nn, 0, -1):
        ijk = stack[ij]
        a[rec[ijk]] = a[rec[ijk]] + a[ijk]
    return a
