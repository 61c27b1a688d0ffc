"""Full-size parity: the first step of the benchmark grids at their full sizes
against digests of the oracle's results (tests/golden/full_size.json, made by
tests/golden/make_full_size.py).

  * closed_basin_8193: 8193x8193, y cyclic, about 1/9 of the nodes pits, so
    LocalMinima dominates (millions of basins, tens of millions of edges);
  * mfd_2049: the 2049x2049 multiple-flow benchmark grid.

Bit-exact: receivers before and after LocalMinima, stack, basin ids, the basin
graph (conn list), its NR sort permutation, the MST in Kruskal's acceptance
order, its orientation, the multiple-flow receivers and their counts.
Floats (h, drainage area, total erosion, basement) on 1024 seeded nodes: within
1e-9 relative (the per-step multiple-flow tolerance of the parity tests).
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX_PATH = os.path.join(HERE, "golden", "full_size.json")
FIX = json.load(open(FIX_PATH)) if os.path.exists(FIX_PATH) else {}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make(case):
    from fastscapelib_fortran import workloads as W
    return {"closed_basin_8193": lambda: W.closed_basin(8193, nsteps=1),
            "mfd_2049": lambda: W.mfd(2049, nsteps=1)}[case]()


@pytest.mark.parametrize("case", sorted(FIX))
def test_first_step_at_full_size(case):
    import torch

    import fastscapelib_fortran as fs

    fx = FIX[case]
    wl = make(case)
    assert (wl.nx, wl.ny) == (fx["nx"], fx["ny"])
    g = fs.FastScape()
    g.set_nx_ny(wl.nx, wl.ny)
    free, _ = torch.cuda.mem_get_info()
    if g.workspace_bytes() > 0.9 * free:
        pytest.skip(f"{case} needs {g.workspace_bytes() / 1e9:.0f} GB of device memory")
    g.setup()
    g.set_xl_yl(wl.xl, wl.yl)
    g.set_dt(wl.dt)
    g.init_h(wl.h0)
    g.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2, wl.p)
    g.set_u(wl.u)
    g.set_bc(wl.bc)
    g.set_capture(True)
    g.execute_step()

    sha = fx["sha256"]
    for f in ("rec_pre", "stack_pre", "basins", "rec", "stack", "mnrec"):
        assert digest(g.copy_int(f).astype(np.int32)) == sha[f], f
    assert digest(g.copy_slots("mrec").astype(np.int32)) == sha["mrec"]
    dbg = g.locmin_debug()
    for k, v in fx["counts"].items():
        assert dbg[k] == v, (k, dbg[k], v)
    for k in ("b1", "b2", "n1", "n2", "w", "sort_id", "tree", "ob1", "ob2", "on1", "on2"):
        assert digest(dbg[k]) == sha["locmin." + k], k

    n = len(fx["sample"]["h"])
    idx = np.sort(np.random.default_rng(fx["sample_index_seed"]).choice(wl.nn, n, replace=False))
    for f, ref in fx["sample"].items():
        out = np.empty(wl.nn)
        g.copy(f, out)
        ref = np.asarray(ref)
        err = np.max(np.abs(out[idx] - ref) / np.maximum(np.abs(ref), 1.0))
        assert err <= 1e-9, (f, err)
    g.destroy()
