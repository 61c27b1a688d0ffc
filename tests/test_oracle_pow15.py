"""How the n = 1.5 powers enter the multiple-flow Newton solves.

The reference evaluates x**1.5 and x**0.5 with pow (StreamPowerLaw.f90:146-162);
the GPU evaluates x*sqrt(x) and sqrt(x), which can differ from pow by an ulp.
The oracle's diagnostic repeats every multiple-flow Newton solve with the GPU's
evaluation on the same inputs and counts the solves whose iteration count or
result differs.

Stated bounds (the benchmark parameters: p = 1.1, n = 1.5, bc 1010): the
iteration count differs in no solve, and a result differs in at most 1e-4 of
the solves, by at most 1e-15 relative.  Measured on the 2049^2 grid over its
first 5 steps: 12,466,315 solves, 1.59 iterations each on average (8 at
most, in the first 3 steps), iteration count never different, 236 results
different (1.9e-5 of the solves), largest difference 3.5e-16 relative.  This
file checks a 257^2 grid.
"""
import oracle as O
from fastscapelib_fortran import workloads as W


def test_pow15_changes_no_iteration_count():
    wl = W.mfd(257, seed=12345)
    wl.apply(O)
    O.pow15_diag(True)
    try:
        for _ in range(3):
            O.fastscape_execute_step()
        d = O.pow15_diag()
    finally:
        O.pow15_diag(False)
        O.fastscape_destroy()
    assert d["solves"] > 100000, d
    assert d["iteration_count_differs"] == 0, d
    assert d["result_differs"] <= 1e-4 * d["solves"], d
    assert d["max_rel_diff"] <= 1e-15, d
    assert d["max_iterations"] <= 20 and d["solves_over_20_iterations"] == 0, d
