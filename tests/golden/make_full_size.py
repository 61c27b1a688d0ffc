"""Writes tests/golden/full_size.json: digests of the oracle's first step on the
full-size benchmark grids, for the GPU parity test at full size.

    python tests/golden/make_full_size.py [case ...]

The oracle (oracle/, the C++ restatement of the reference) runs one
FastScape_Execute_Step on each grid; the fixture keeps, per case, the SHA-256
of every integer artefact of the step (receivers before and after
LocalMinima, stack, basin ids, the basin graph, its NR sort permutation, the
MST in acceptance order and its orientation, the multiple-flow receivers)
and a seeded sample of 1024 nodes of the float64 outputs.  Integer artefacts
must match bit for bit; floats within the per-step tolerance of the parity
tests.  Cases: closed_basin_8193 (8193x8193, ~25 GB of host memory, about two
minutes) and mfd_2049 (2049x2049).
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "fastscapelib-fortran_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

INT_FIELDS = ("rec_pre", "stack_pre", "basins", "rec", "stack", "mnrec")
LOCMIN = ("b1", "b2", "n1", "n2", "w", "sort_id", "tree", "ob1", "ob2", "on1", "on2")
LOCMIN_COUNTS = ("nbasins", "basin0", "nconn", "tree_size", "nlocmin_before", "nlocmin_after")
FLOAT_FIELDS = ("h", "drainage_area", "total_erosion", "basement")
SAMPLE = 1024
SAMPLE_SEED = 2024


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    from fastscapelib_fortran import workloads as W
    return {"closed_basin_8193": lambda: W.closed_basin(8193, nsteps=1),
            "mfd_2049": lambda: W.mfd(2049, nsteps=1)}


def sample_index(nn: int) -> np.ndarray:
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(nn, SAMPLE, replace=False))


def run_case(make):
    import oracle as O
    wl = make()
    t0 = time.time()
    wl.apply(O)
    O.fastscape_execute_step()
    out = {"workload": wl.name, "nx": wl.nx, "ny": wl.ny, "steps": 1, "sha256": {}}
    for f in INT_FIELDS:
        out["sha256"][f] = digest(O.copy_int(f).astype(np.int32))
    out["sha256"]["mrec"] = digest(O.copy_slots("mrec").astype(np.int32))
    dbg = O.locmin_debug()
    for k in LOCMIN:
        out["sha256"]["locmin." + k] = digest(dbg[k])
    out["counts"] = {k: int(dbg[k]) for k in LOCMIN_COUNTS}
    idx = sample_index(wl.nn)
    out["sample_index_seed"] = SAMPLE_SEED
    out["sample"] = {f: O.copy_double(f)[idx].tolist() for f in FLOAT_FIELDS}
    out["oracle_seconds"] = round(time.time() - t0, 1)
    O.fastscape_destroy()
    return out


def main():
    path = os.path.join(HERE, "full_size.json")
    data = json.load(open(path)) if os.path.exists(path) else {}
    want = sys.argv[1:] or list(cases())
    for name, make in cases().items():
        if name in want:
            data[name] = run_case(make)
            print(name, data[name]["counts"], data[name]["oracle_seconds"], "s", flush=True)
            json.dump(data, open(path, "w"), indent=1)


if __name__ == "__main__":
    main()
