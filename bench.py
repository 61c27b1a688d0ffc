"""Benchmark of the continental time step (node-steps/s) on B200.

Default workload: the 2049x2049 multiple-flow grid (xl=yl=200 km, bc=1010,
p=1.1, n=1.5 Newton, kf=2e-6, m=0.45, kd=5e-2, dt=500, h=U[0,10)+1e-3*j,
interior uplift 5e-4), seeded synthetic input.  A step is one
FastScape_Execute_Step of that grid; the timed steps follow W warm-up steps of
the same trajectory.  The grid's working set (~4 GB) is far larger than the
126 MB L2, so no explicit L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Two more workloads (one GPU, reported on their own JSON line):

    python bench.py --workload batched   # 256 uneven single-flow grids, 100 steps each,
                                         # run concurrently by a Batch (fsb_batch_*)
    python bench.py --workload served    # multiple-flow requests with Poisson arrivals at
                                         # five rates: p50/p99 latency and node-steps/s

Multi-GPU runs are independent replicas (one instance per GPU, no collective):
a single grid's routing tree, basin graph and implicit solves are global
dependencies, so the path does not shard; value = nodes*steps of all ranks /
max time over ranks ("scaling": "weak").

--impl reference times the reference's CPU algorithm: the C++ restatement in
oracle/ (the Fortran reference cannot be compiled here), one single-threaded
instance per host core, each stepping the same workload.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fastscapelib-fortran_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "node-steps/s at 2049^2 (continental step, MFD p=1.1, n=1.5, FP64)"
UNIT = "node-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=2049)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--workload", default="mfd", choices=["mfd", "batched", "served"])
    ap.add_argument("--workers", type=int, default=32, help="batch worker streams")
    ap.add_argument("--grids", type=int, default=256, help="batched: number of grids")
    ap.add_argument("--job-steps", type=int, default=100, help="batched: steps per grid")
    ap.add_argument("--requests", type=int, default=100, help="served: requests per rate")
    ap.add_argument("--probe-requests", type=int, default=24,
                    help="served: requests submitted at once to measure the capacity")
    ap.add_argument("--loads", default="0.5,0.7,0.85,1.0,1.2",
                    help="served: arrival rates as fractions of the measured capacity")
    ap.add_argument("--precision", default="fp64", help="served/batched: fp64, mixed or fp64,mixed")
    ap.add_argument("--mixed-loads", default=None,
                    help="served: loads for the mixed form (default: --loads)")
    ap.add_argument("--step-scale", type=float, default=1.0,
                    help="served: scale of the 20..400 steps per request (1 = as specified)")
    ap.add_argument("--max-side", type=int, default=4097, help="served: largest grid side")
    ap.add_argument("--mem-budget", type=float, default=150e9, help="device bytes for jobs")
    return ap.parse_args()


def workloads_module():
    """The synthetic-workload generators, loaded from their file on their own.

    Importing them through the package would run its __init__, which maps
    the CUDA library; the reference arm (oracle only) must not load it."""
    import importlib.util
    name = "fsb_workloads_standalone"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "fastscapelib-fortran_b200", "fastscapelib_fortran", "workloads.py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(size, seed=12345):
    return workloads_module().mfd(size, seed=seed)


def clocks_path(name):
    """Where a run's sampled clock log goes: $FSB_CLOCKS_DIR if set, else the
    temporary directory (the JSON line carries the summary either way)."""
    return os.path.join(os.environ.get("FSB_CLOCKS_DIR") or tempfile.gettempdir(), name)


def l2_note(nodes):
    """How the timed steps stand against the 126 MB L2: the instance's arena
    is about 1.1 KB per node and every step sweeps all of it."""
    ws = 1100.0 * nodes
    if ws > 4 * 126e6:
        return "working set %.1f GB >> 126 MB L2 (no flush needed)" % (ws / 1e9)
    return "working set %.0f MB, not flushed between steps (small case; not a bench configuration)" % (ws / 1e6)


def config(args, wl, ranks):
    return {"workload": f"mfd_{wl.nx}x{wl.ny}_bc{wl.bc}_p{wl.p}_n{wl.n}", "nx": wl.nx, "ny": wl.ny,
            "grids_per_gpu": 1, "parallelism": f"replicas{ranks}" if ranks > 1 else "single",
            "l2": l2_note(wl.nx * wl.ny)}


# ---------------------------------------------------------------------------
# oracle (CPU) timing

def _oracle_worker(args):
    size, seed, warm, steps = args
    import oracle as O
    wl = workload(size, seed)
    wl.apply(O)
    for _ in range(warm):
        O.fastscape_execute_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        O.fastscape_execute_step()
    return time.perf_counter() - t0, wl.nn * steps


def cpu_baseline(size, steps):
    t, nodes = _oracle_worker((size, 12345, 0, steps))
    return {"value": nodes / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {steps} steps of the {size}x{size} workload, C++ restatement of the "
                      f"reference (oracle/), 1 thread, {t:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # one single-threaded instance per host core, as many as host memory allows
    # (about 2.5 GB per 2049^2 instance); each needs ~4 s per 2049^2 step
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil
        mem_cap = int(psutil.virtual_memory().available / (2.5e9 * (args.size / 2049.0) ** 2))
    except Exception:
        mem_cap = cores
    procs = max(1, min(cores, mem_cap))
    jobs = [(args.size, 12345 + r, args.warmup, args.steps) for r in range(procs)]
    t0 = time.perf_counter()
    if procs > 1:
        # instances 1..procs-1 in spawned workers, instance 0 in this process
        with mp.get_context("spawn").Pool(procs - 1) as pool:
            pending = pool.map_async(_oracle_worker, jobs[1:])
            res = [_oracle_worker(jobs[0])] + pending.get()
    else:
        res = [_oracle_worker(jobs[0])]
    wall = time.perf_counter() - t0
    tmax = max(t for t, _ in res)
    nodes = sum(n for _, n in res)
    value = nodes / tmax
    wl = workload(args.size)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tmax / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(args, wl, 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                             "sample": f"{procs} independent single-threaded instances x "
                                       f"{args.steps} steps after {args.warmup} warm-up steps "
                                       f"({wall:.0f} s wall)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# ranks: independent replicas, one per GPU, timed as the slowest rank

def max_over_ranks(times_ms, device, world):
    """Every rank's times, reduced with MAX over the process group (world > 1)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in times_ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    return [float(x) for x in t]


def replica_throughput(nn, steps, world, ms_max):
    """Whole-job node-steps/s: every rank stepped its own nn-node grid `steps`
    times; the job took as long as the slowest rank."""
    return nn * steps * world / (ms_max / 1e3)


# ---------------------------------------------------------------------------
# GPU arm

class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index, path):
        self.path = path
        self.proc = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sms:
            return None
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


# algorithmic bytes per node of each stage (FP64 values, int32 indices; rbar =
# mean number of multiple-flow receivers, nconn = basin-graph edges)
def stage_bytes(stage, rbar, nconn_per_node, sfd):
    table = {
        "uplift": 40.0,
        "receivers": 20.0,
        "stack": 16.0,
        "local_minima": 52.0 + 48.0 * nconn_per_node,
        "lake_fill": 32.0,
        "mfd_receivers": 12.0 + 20.0 * rbar,
        "drainage_area": 24.0 if sfd else 16.0 + 12.0 * rbar,
        "stream_power": 88.0 if sfd else 88.0 + 20.0 * rbar,
        "diffusion": 88.0,
    }
    return table[stage]


def measured_traffic(kernel, nn):
    """DRAM bytes per launch of `kernel` (dram__bytes_read.sum + _write.sum),
    scaled to nn nodes from the per-node figure of the ncu capture committed in
    profiles/kernel_traffic.json -- but only while the kernel's source file is
    the one that capture measured (SHA-256 recorded beside the figure)."""
    import hashlib
    path = os.path.join(ROOT, "profiles", "kernel_traffic.json")
    if not os.path.exists(path):
        return None, "no capture committed"
    rec = json.load(open(path)).get(kernel)
    if rec is None:
        return None, "no capture of this kernel"
    src = os.path.join(ROOT, rec["source"])
    sha = hashlib.sha256(open(src, "rb").read()).hexdigest()
    if sha != rec["source_sha256"]:
        return None, f"capture of an earlier {rec['source']} (source changed since)"
    return rec["bytes_per_node"] * nn, f"{rec['capture']}, scaled by nodes"


def run_gpu(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import fastscapelib_fortran as fs

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.size, args.cpu_steps)

    wl = workload(args.size, seed=12345 + rank)
    g = fs.FastScape(local)
    g.set_nx_ny(wl.nx, wl.ny)
    g.setup()
    g.set_xl_yl(wl.xl, wl.yl)
    g.set_dt(wl.dt)
    g.init_h(wl.h0)
    g.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2, wl.p)
    g.set_u(wl.u)
    g.set_bc(wl.bc)
    stream = torch.cuda.current_stream(dev)

    for _ in range(args.warmup):
        g.execute_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    # timed region: K steps with stage profiling off
    clocks = ClockSampler(local, clocks_path(f"clocks_r{rank}.csv"))
    launches0 = g.launch_count()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.execute_step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    launches = g.launch_count() - launches0

    # the FP64 surface after W + K steps, the reference for the mixed form
    h_fp64 = torch.empty(wl.nn, dtype=torch.float64, device=dev)
    g.copy("h", h_fp64)
    torch.cuda.synchronize()
    mixed = None
    if world == 1:
        mixed = run_mixed(args, wl, local, stream, h_fp64, ms / args.steps)

    # a separate pass of K more steps with per-stage CUDA events (not part of
    # the timed region: the events and their read-backs cost time)
    g.set_profile(True)
    g.stage_times(reset=True)
    g.execute_step(args.steps)
    torch.cuda.synchronize()
    stages = g.stage_times(reset=True)
    g.set_profile(False)

    # e2e through the reference-facing API with host buffers: set_u from pinned
    # host memory, execute_step, copy_h back into pinned host memory
    u_host = torch.from_numpy(wl.u.copy()).pin_memory()
    h_host = torch.empty(wl.nn, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        g.set_u(u_host)
        g.execute_step()
        g.copy("h", h_host)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(f0.elapsed_time(f1), 1e3 * (time.perf_counter() - t0))

    ms_max, e2e_max = max_over_ranks([ms, e2e_ms], dev, world)
    value = replica_throughput(wl.nn, args.steps, world, ms_max)
    e2e_val = replica_throughput(wl.nn, args.steps, world, e2e_max)

    if rank == 0:
        mnrec = g.copy_int("mnrec")
        rbar = float(mnrec.mean())
        dbg_nconn = g.locmin_debug()["nconn"]
        # the dominant single kernel among the timed ones, with the algorithmic
        # bytes of the stage it carries (the sweep kernels do that stage's work)
        kstage = {"k_spl_sweep": "stream_power", "k_area_sweep": "drainage_area",
                  "k_fill_chains": "lake_fill", "k_thomas_rows": "diffusion", "k_thomas_cols": "diffusion"}
        ktimes = {k: v for k, v in stages.items() if k in kstage and v[1]}
        name, (tot_ms, calls) = max(ktimes.items(), key=lambda kv: kv[1][0] / max(kv[1][1], 1))
        per_launch_ms = tot_ms / max(calls, 1)
        bpn = stage_bytes(kstage[name], rbar, dbg_nconn / wl.nn, wl.p < -1.5)
        if name.startswith("k_thomas"):
            bpn /= 2.0  # one of the two line passes of the diffusion
        achieved = bpn * wl.nn / (per_launch_ms / 1e3) / 1e9
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        peak, peak_src = 6650.0, "fallback"
        if os.path.exists(peaks_path):
            peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
        traffic, traffic_note = measured_traffic(name, wl.nn)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(args, wl, world),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 8 * wl.nn,
                    "d2h_bytes_per_step": 8 * wl.nn},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                         "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": traffic_note,
                         "bytes_per_node": bpn, "launch_ms": per_launch_ms},
            "stages_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in stages.items()
                                   if not k.startswith("k_")},
            "kernels_ms_per_launch": {k: v[0] / max(v[1], 1) for k, v in stages.items()
                                      if k.startswith("k_") and v[1]},
            "clocks": clk,
            "cpu_baseline": cpu,
            "mixed": mixed,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_mixed(args, wl, local, stream, h_fp64, fp64_ms_per_step):
    """The same workload in the mixed-precision form: W warm-up and K timed
    steps (CUDA events on the instance's stream), then the surface compared
    with the FP64 form's after the same W + K steps."""
    import torch
    import fastscapelib_fortran as fs
    gm = fs.FastScape(local)
    gm.set_nx_ny(wl.nx, wl.ny)
    gm.setup()
    gm.set_precision("mixed")
    gm.set_xl_yl(wl.xl, wl.yl)
    gm.set_dt(wl.dt)
    gm.init_h(wl.h0)
    gm.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2, wl.p)
    gm.set_u(wl.u)
    gm.set_bc(wl.bc)
    for _ in range(args.warmup):
        gm.execute_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    gm.execute_step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    hm = torch.empty_like(h_fp64)
    gm.copy("h", hm)
    torch.cuda.synchronize()
    err = float(((hm - h_fp64).abs() / h_fp64.abs().clamp(min=1.0)).max())
    gm.destroy()
    value = wl.nn * args.steps / (ms / 1e3)
    return {"value": value, "unit": UNIT, "ms_per_step": ms / args.steps,
            "dtype": "mixed: fp32 weights, area, Newton increments, tridiagonal increments; "
                     "fp64 state, h update, residuals; exact routing",
            "speedup_vs_fp64": fp64_ms_per_step / (ms / args.steps),
            "h_rel_linf_vs_fp64": err, "after_steps": args.warmup + args.steps}


# ---------------------------------------------------------------------------
# many grids on one GPU: batched and served forms

def _batch_cpu_sample(wls, seconds=10.0):
    """The oracle (1 thread) on the first grids of a list, two steps each."""
    import oracle as O
    t = nodes = 0.0
    used = 0
    for w in wls:
        w.apply(O)
        t0 = time.perf_counter()
        for _ in range(2):
            O.fastscape_execute_step()
        t += time.perf_counter() - t0
        nodes += 2 * w.nn
        used += 1
        if t > seconds:
            break
    return {"value": nodes / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {used} grids x 2 steps, C++ restatement of the reference (oracle/), "
                      f"1 thread, {t:.1f} s"}


def run_batched(args):
    import numpy as np
    import torch
    import fastscapelib_fortran as fs
    from fastscapelib_fortran import workloads as W

    torch.cuda.set_device(0)
    wls = W.uneven_d8(args.grids, nsteps=args.job_steps)
    cpu = None if args.no_cpu_baseline else _batch_cpu_sample(wls)
    # the work table is submitted largest grid first, so that no large grid
    # starts last and runs alone at the end
    wls.sort(key=lambda w: -w.nn * w.nsteps)
    node_steps = sum(w.nn * w.nsteps for w in wls)
    forms = {}
    precs = args.precision.split(",")
    clocks = ClockSampler(0, clocks_path("clocks_batched.csv"))
    with fs.Batch(workers=args.workers, mem_budget=int(args.mem_budget)) as b:
        for prec in precs:
            # warm-up: one small job per worker (library, streams, memory pool)
            b.run([w.job(precision=prec) for w in W.uneven_d8(args.workers, seed=999,
                                                              nsteps=max(args.warmup, 1),
                                                              lo=129, hi=257)])
            jobs = [w.job(precision=prec) for w in wls]
            t0 = time.perf_counter()
            b.run(jobs)
            wall = time.perf_counter() - t0
            lat = np.array([j.t_end - j.t_submit for j in jobs])
            forms[prec] = {"value": node_steps / wall, "wall_s": wall,
                           "job_latency_s": {"p50": float(np.percentile(lat, 50)),
                                             "p99": float(np.percentile(lat, 99))}}
    clk = clocks.stop()
    sides = np.array([w.nx for w in wls])
    value = forms[precs[0]]["value"]
    lat = np.array([forms[precs[0]]["job_latency_s"]["p50"], forms[precs[0]]["job_latency_s"]["p99"]])
    line = {
        "metric": "node-steps/s, 256 uneven single-flow grids run concurrently",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.job_steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": f"uneven_d8 x{len(wls)} (sides {sides.min()}..{sides.max()}, "
                               f"{args.job_steps} steps each, bc=1111, p=-2, per-grid kf,m,n,kd,U)",
                   "grids": len(wls), "total_nodes": int(sum(w.nn for w in wls)),
                   "workers": args.workers, "order": "largest first",
                   "timing": "host wall clock, first submit to last result",
                   "l2": "working set >> 126 MB L2"},
        "e2e": {"value": value, "unit": UNIT,
                "h2d_bytes_per_step": int(sum(4 * 8 * w.nn for w in wls)) // args.job_steps,
                "d2h_bytes_per_step": int(sum(8 * w.nn for w in wls)) // args.job_steps},
        "job_latency_s": {"p50": float(lat[0]), "p99": float(lat[1])}, "forms": forms,
        "clocks": clk, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_served(args):
    import threading

    import numpy as np
    import torch
    import fastscapelib_fortran as fs
    from fastscapelib_fortran import workloads as W

    torch.cuda.set_device(0)
    scale = args.step_scale
    steps = (max(1, int(round(20 * scale))), max(1, int(round(400 * scale))))

    def requests(seed):
        return W.served_mfd(args.requests, seed=seed, hi=args.max_side, steps=steps)

    def serve(b, reqs, rate, rng, prec="fp64"):
        """Submits at Poisson arrival times; returns (latencies, node-steps/s)."""
        gaps = rng.exponential(1.0 / rate, len(reqs)) if rate > 0 else np.zeros(len(reqs))
        arrivals = np.cumsum(gaps) - gaps[0]
        ids = [None] * len(reqs)
        jobs = [r.job(precision=prec) for r in reqs]
        t0 = time.perf_counter()

        def submitter():
            for k, job in enumerate(jobs):
                dt = t0 + arrivals[k] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[k] = b.submit(job)

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for jid in ids:
            b.wait(jid)
        span = max(j.t_end for j in jobs) - min(j.t_submit for j in jobs)
        lat = np.array([j.t_end - j.t_submit for j in jobs])
        return lat, sum(r.nn * r.nsteps for r in reqs) / span

    forms = {}
    clocks = ClockSampler(0, clocks_path("clocks_served.csv"))
    with fs.Batch(workers=args.workers, mem_budget=int(args.mem_budget)) as b:
        for prec in args.precision.split(","):
            b.run([w.job(precision=prec) for w in W.served_mfd(args.workers, seed=999, hi=513,
                                                                steps=(2, 2))])
            # capacity: a probe set of requests submitted at once
            probe = W.served_mfd(args.probe_requests, seed=777, hi=args.max_side, steps=steps)
            _, thr = serve(b, probe, 0.0, np.random.default_rng(0), prec)
            work = np.mean([r.nn * r.nsteps for r in probe])
            mu = thr / work  # requests per second the GPU completes when saturated
            loads = args.loads if prec == "fp64" or not args.mixed_loads else args.mixed_loads
            levels = []
            for lv, frac in enumerate(float(x) for x in loads.split(",")):
                rate = frac * mu
                lat, thr = serve(b, requests(1000 + lv), rate, np.random.default_rng(lv), prec)
                levels.append({"rate_per_s": rate, "load": frac, "requests": len(lat),
                               "p50_s": float(np.percentile(lat, 50)),
                               "p99_s": float(np.percentile(lat, 99)),
                               "max_s": float(lat.max()), "node_steps_per_s": thr})
            forms[prec] = {"capacity_req_per_s": mu, "probe_node_steps_per_s": mu * work,
                           "levels": levels}
    clk = clocks.stop()
    first = forms[args.precision.split(",")[0]]
    top = max(first["levels"], key=lambda lv: lv["node_steps_per_s"])
    line = {
        "metric": "served multiple-flow requests: p50/p99 latency (s) and node-steps/s",
        "value": top["node_steps_per_s"], "unit": UNIT, "n_gpus": 1, "steps": None,
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {"workload": f"served_mfd: sides log-uniform 257..{args.max_side} (odd), steps "
                               f"uniform {steps[0]}..{steps[1]}, p=1.1, n=1.5, bc=1010, "
                               f"{args.requests} Poisson requests per rate",
                   "loads": args.loads, "workers": args.workers, "mem_budget": args.mem_budget,
                   "timing": "host wall clock from each arrival to its result"},
        "e2e": {"value": top["node_steps_per_s"], "unit": UNIT, "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None},
        "forms": forms, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "batched":
        run_batched(args)
    elif args.workload == "served":
        run_served(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
