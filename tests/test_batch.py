"""Many grids on one device (fsb_batch_* through fastscapelib_fortran.Batch).

Checked here:
  * a job's results are bit-identical whether it runs alone on a FastScape
    instance, alone in a one-worker batch, or in a mix of uneven single- and
    multiple-flow jobs on several workers (the kernels' arithmetic is fixed per
    node, so nothing that runs beside a job can change it);
  * batch results against the oracle: single flow within 1e-10 relative after
    three free-running steps (1e-12 per step, see the parity tests);
  * admission by device memory: with a budget that holds one job at a time the
    jobs still all complete, correctly; a job larger than the budget is refused;
  * a failing job reports its error without disturbing the others;
  * continuous batching: a job submitted while others are on the GPU (the
    served form's admission) gives the same bits as alone, in FP64 and in the
    mixed-precision form.
"""
import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

pytestmark = pytest.mark.gpu


def mix():
    return [W.plain_d8(33, 29, seed=1, nsteps=4), W.mfd(41, 37, seed=2, nsteps=3),
            W.plain_d8(65, 65, seed=3, nsteps=2), W.mfd(29, 57, seed=4, nsteps=4, n=1.0, p=0.0),
            W.uneven_d8(2, seed=5, nsteps=3, lo=129, hi=161)[1],
            W.plain_d8(47, 31, seed=6, nsteps=5, p=-2.0)]


def alone(wl, precision="fp64"):
    import fastscapelib_fortran as fs
    g = fs.FastScape()
    g.set_nx_ny(wl.nx, wl.ny)
    g.setup()
    g.set_precision(precision)
    g.set_xl_yl(wl.xl, wl.yl)
    g.set_dt(wl.dt)
    g.init_h(wl.h0.copy())
    g.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2, wl.p)
    g.set_u(wl.u)
    g.set_bc(wl.bc)
    g.execute_step(wl.nsteps)
    h, a = np.empty(wl.nn), np.empty(wl.nn)
    g.copy("h", h)
    g.copy("drainage_area", a)
    g.destroy()
    return h, a


def test_same_alone_and_in_the_mix():
    import fastscapelib_fortran as fs
    wls = mix()
    ref = [alone(w) for w in wls]
    with fs.Batch(workers=1) as b:
        serial = b.run([w.job(want_area=True) for w in wls])
    with fs.Batch(workers=4) as b:
        mixed = b.run([w.job(want_area=True) for w in wls] * 2)
    for k, w in enumerate(wls):
        for jobs in (serial, mixed[:len(wls)], mixed[len(wls):]):
            assert np.array_equal(jobs[k].h, ref[k][0]), w.name
            assert np.array_equal(jobs[k].a, ref[k][1]), w.name
        assert mixed[k].t_submit <= mixed[k].t_start <= mixed[k].t_end


def test_batch_against_oracle():
    import fastscapelib_fortran as fs
    wls = [W.plain_d8(37, 33, seed=7, nsteps=3), W.plain_d8(25, 41, seed=8, nsteps=3)]
    with fs.Batch(workers=2) as b:
        jobs = b.run([w.job() for w in wls])
    for w, j in zip(wls, jobs):
        w.apply(O)
        for _ in range(w.nsteps):
            O.fastscape_execute_step()
        ho = O.copy_double("h")
        err = np.max(np.abs(j.h - ho) / np.maximum(np.abs(ho), 1.0))
        assert err <= 1e-10, (w.name, err)


def test_admission_by_memory():
    import fastscapelib_fortran as fs
    wls = [W.plain_d8(65, 65, seed=s, nsteps=2) for s in range(4)]
    g = fs.FastScape()
    g.set_nx_ny(65, 65)
    one = g.workspace_bytes()
    g.destroy()
    ref = [alone(w)[0] for w in wls]
    with fs.Batch(workers=4, mem_budget=int(one * 1.5) + (2 << 20)) as b:
        jobs = b.run([w.job() for w in wls])
        assert b.memory()["in_use"] == 0
        # one at a time: no job started before the previous one ended
        spans = sorted((j.t_start, j.t_end) for j in jobs)
        for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
            assert s1 >= e0
        with pytest.raises(RuntimeError, match="budget"):
            b.submit(W.plain_d8(257, 257, seed=1, nsteps=1).job())
    for j, r in zip(jobs, ref):
        assert np.array_equal(j.h, r)


def test_failing_job_is_isolated():
    import fastscapelib_fortran as fs
    good = W.plain_d8(33, 33, seed=9, nsteps=2)
    bad = W.plain_d8(33, 33, seed=9, nsteps=2)
    bad.bc = 0  # no fixed boundary: LocalMinima has no outlet, the job must fail
    with fs.Batch(workers=2) as b:
        ids = [b.submit(good.job()), b.submit(bad.job()), b.submit(good.job())]
        j0 = b.wait(ids[0])
        with pytest.raises(RuntimeError):
            b.wait(ids[1])
        j2 = b.wait(ids[2])
    ref = alone(good)[0]
    assert np.array_equal(j0.h, ref) and np.array_equal(j2.h, ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_submitted_while_others_run(precision):
    """Requests that arrive while others are running are admitted and overlap
    with them on the device; each result equals its solo run bit for bit."""
    import time

    import fastscapelib_fortran as fs
    long_jobs = [W.mfd(257, 257, seed=20 + k, nsteps=30) for k in range(3)]
    late = [W.mfd(129, 121, seed=30, nsteps=6), W.plain_d8(97, 89, seed=31, nsteps=6)]
    ref = [alone(w, precision)[0] for w in late]
    with fs.Batch(workers=4) as b:
        first = [b.submit(w.job(precision=precision)) for w in long_jobs]
        t0 = time.perf_counter()
        while b.memory()["running"] == 0 and time.perf_counter() - t0 < 60:
            time.sleep(0.001)
        assert b.memory()["running"] > 0
        ids = [b.submit(w.job(precision=precision)) for w in late]
        done_late = [b.wait(i) for i in ids]
        done_first = [b.wait(i) for i in first]
    # the late jobs started while a long job was still running
    assert min(j.t_start for j in done_late) < max(j.t_end for j in done_first)
    for j, r in zip(done_late, ref):
        assert np.array_equal(j.h, r)
