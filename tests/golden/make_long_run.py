"""Writes tests/golden/long_run.json: the oracle's state after many free-running
steps of the benchmark grids, for the GPU test of the error after N steps.

    python tests/golden/make_long_run.py [case ...]

The oracle (oracle/, the C++ restatement of the reference) steps each grid
from its seeded initial surface without any re-synchronisation and, at each
checkpoint, keeps a seeded sample of 2048 nodes of every float64 output and
the min / mean / max of each full field.  Cases:

  * mfd_2049: the 2049x2049 multiple-flow benchmark grid (p = 1.1, n = 1.5
    Newton, bc = 1010), checkpoints after 20, 100 and 500 steps -- the full
    length of that configuration; about 35 minutes of oracle time;
  * plain_101_p0: the 101x101 configuration read literally (p = 0, uniform
    multiple flow), checkpoints after 50 and 200 steps.

The GPU test (tests/test_long_runs.py) runs the same steps and reports the
relative L-infinity error per field on the sample.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "fastscapelib-fortran_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

FIELDS = ("h", "drainage_area", "total_erosion", "erosion_rate", "basement", "lake_depth")
SAMPLE = 2048
SAMPLE_SEED = 4242


def load_workloads():
    """The workload generators without importing the package (which maps the
    CUDA library)."""
    import importlib.util
    name = "fsb_workloads_fixture"
    path = os.path.join(ROOT, "fastscapelib-fortran_b200", "fastscapelib_fortran", "workloads.py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def cases():
    W = load_workloads()
    return {"mfd_2049": (lambda: W.mfd(2049, nsteps=500), (20, 100, 500)),
            "plain_101_p0": (lambda: W.plain_d8(101, nsteps=200, p=0.0), (50, 200))}


def sample_index(nn: int) -> np.ndarray:
    n = min(SAMPLE, nn)
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(nn, n, replace=False))


def run_case(make, checkpoints):
    import oracle as O
    wl = make()
    t0 = time.time()
    wl.apply(O)
    idx = sample_index(wl.nn)
    out = {"workload": wl.name, "nx": wl.nx, "ny": wl.ny, "p": wl.p, "bc": wl.bc,
           "sample_index_seed": SAMPLE_SEED, "sample_size": int(len(idx)), "checkpoints": {}}
    step = 0
    for cp in checkpoints:
        while step < cp:
            O.fastscape_execute_step()
            step += 1
        rec = {"sample": {}, "stats": {}}
        for f in FIELDS:
            v = O.copy_double(f)
            rec["sample"][f] = v[idx].tolist()
            rec["stats"][f] = [float(v.min()), float(v.mean()), float(v.max())]
        out["checkpoints"][str(cp)] = rec
        print(wl.name, "step", cp, round(time.time() - t0, 1), "s", flush=True)
    out["oracle_seconds"] = round(time.time() - t0, 1)
    O.fastscape_destroy()
    return out


def main():
    path = os.path.join(HERE, "long_run.json")
    data = json.load(open(path)) if os.path.exists(path) else {}
    want = sys.argv[1:] or list(cases())
    for name, (make, cps) in cases().items():
        if name in want:
            data[name] = run_case(make, cps)
            json.dump(data, open(path, "w"), indent=0)


if __name__ == "__main__":
    main()
