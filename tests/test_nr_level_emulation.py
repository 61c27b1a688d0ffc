"""The level-synchronous emulation of the NR index sort, on the CPU.

The GPU reproduces loc_min_3_indexx (LocalMinima.f90:947-1046) without
running its quicksort sequentially: every partition of a level is rebuilt
from the positions of the Hoare scans' stoppers (prefix sums) and a crossing
rule (nr_cross_one), then segments of 8..512 elements are finished in shared
memory (nr_sort_local) and smaller ones by straight insertion.  The per-level
functions are plain C++ apart from two atomics, so this test compiles them
from csrc/fsb_locmin.cu for the host with g++, drives the same level loop
sequentially (the launch-per-level path of nr_indexx, one position or segment
at a time) and checks the permutation against the oracle's sequential sort,
ties included, on sizes that take many levels.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "fastscapelib-fortran_b200", "csrc", "fsb_locmin.cu")

DRIVER = r"""
#include <algorithm>
#include <utility>
#include <vector>
using std::max;
using std::min;
static inline int atomicAdd(int* p, int v) { const int o = *p; *p += v; return o; }
static inline int atomicExch(int* p, int v) { const int o = *p; *p = v; return o; }
%(enum)s
%(consts)s
%(level_functions)s
%(sort_local)s

// the level loop of nr_indexx with every kernel run over its range in order
extern "C" int nr_emulate(int n, const double* w, int* perm, int* levels_out) {
  const double* arr = w - 1;  // 1-based
  const int cap = n + 16;
  std::vector<int> idx(n + 2), idx2(n + 2), segof(n + 2), lf(n + 2), rf(n + 2), ls(n + 2), rs(n + 2),
      lpos(n + 2), rpos(n + 2), seg(2 * cap), seg2(2 * cap), meta(4 * cap), small(2 * cap), med(2 * cap);
  std::vector<double> piv(cap);
  int cnt[32] = {0};
  const bool level = n > kNrMedium;  // k_nr_init
  for (int q = 0; q <= n + 1; ++q) {
    idx[q] = (q >= 1 && q <= n) ? q : 0;
    segof[q] = (q >= 1 && q <= n && level) ? 0 : -1;
  }
  if (level) { seg[0] = 1; seg[1] = n; cnt[C_NSEG] = 1; }
  else if (n - 1 >= 7) { med[0] = 1; med[1] = n; cnt[C_NMED] = 1; }
  else if (n >= 2) { small[0] = 1; small[1] = n; cnt[C_NSMALL] = 1; }
  int in = C_NSEG, out = C_NSEG2, levels = 0;
  while (cnt[in] > 0) {
    if (++levels > nr_max_levels(n)) return -1;
    const int nseg = cnt[in];
    for (int s = 0; s < nseg; ++s) nr_median_one(s, seg.data(), arr, idx.data(), piv.data(), meta.data());
    for (int q = 0; q <= n + 1; ++q) {
      int a, b;
      nr_flags_one(q, segof.data(), seg.data(), piv.data(), arr, idx.data(), a, b);
      lf[q] = a;
      rf[q] = b;
    }
    int sl = 0, sr = 0;  // exclusive scans and the stopper positions (k_nr_scatter)
    for (int q = 0; q <= n + 1; ++q) { ls[q] = sl; rs[q] = sr; sl += lf[q]; sr += rf[q]; }
    for (int q = 0; q <= n + 1; ++q) {
      if (lf[q]) lpos[ls[q]] = q;
      if (rf[q]) rpos[rs[q]] = q;
    }
    for (int s = 0; s < nseg; ++s)
      nr_cross_one(s, seg.data(), ls.data(), rs.data(), lpos.data(), rpos.data(), meta.data());
    for (int q = 1; q <= n; ++q)
      idx2[q] = nr_apply_one(q, segof.data(), seg.data(), meta.data(), idx.data(), lf.data(), rf.data(),
                             ls.data(), rs.data(), lpos.data(), rpos.data());
    std::swap(idx, idx2);
    cnt[out] = 0;
    for (int s = 0; s < nseg; ++s)
      nr_newsegs_one(s, out, seg.data(), meta.data(), meta.data(), seg2.data(), small.data(), med.data(), cnt, cap, cap);
    for (int q = 0; q <= n + 1; ++q) nr_segof_one(q, seg.data(), meta.data(), segof.data());
    std::swap(seg, seg2);
    std::swap(in, out);
  }
  for (int m = 0; m < cnt[C_NMED]; ++m) {  // k_nr_medium
    const int l = med[2 * m], len = med[2 * m + 1] - l + 1;
    std::vector<double> key(len);
    std::vector<int> id(len);
    for (int p = 0; p < len; ++p) { id[p] = idx[l + p]; key[p] = arr[id[p]]; }
    if (!nr_sort_local(key.data(), id.data(), len)) return -2;
    for (int p = 0; p < len; ++p) idx[l + p] = id[p];
  }
  for (int s = 0; s < cnt[C_NSMALL]; ++s) {  // k_nr_insertion
    const int l = small[2 * s], ir = small[2 * s + 1];
    for (int j = l + 1; j <= ir; ++j) {
      const int indxt = idx[j];
      const double a = arr[indxt];
      int i = j - 1;
      for (; i >= l; --i) {
        if (arr[idx[i]] <= a) break;
        idx[i + 1] = idx[i];
      }
      idx[i + 1] = indxt;
    }
  }
  for (int t = 0; t < n; ++t) perm[t] = idx[t + 1] - 1;
  *levels_out = levels;
  return cnt[C_OVERFLOW];
}
"""


def _between(text, start, end_marker, include_end=True):
    i = text.index(start)
    j = text.index(end_marker, i)
    return text[i:j + (len(end_marker) if include_end else 0)]


def _function(text, signature):
    i = text.index(signature)
    return text[i:text.index("\n}\n", i) + 3]


@pytest.fixture(scope="module")
def emulate(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    text = open(SRC).read()
    enum = _between(text, "enum {\n  C_NBASINS", "};")
    consts = "\n".join(l for l in text.splitlines()
                       if l.startswith("constexpr int kNrCounters") or l.startswith("constexpr int kNrMedium")
                       or l.startswith("inline int nr_max_levels"))
    levels = _between(text, "__device__ inline void iswap", "__device__ inline void nr_segof_one", False)
    levels += _function(text, "__device__ inline void nr_segof_one")
    sort_local = _function(text, "__device__ bool nr_sort_local(")
    src = DRIVER % {"enum": enum, "consts": consts, "level_functions": levels.replace("__device__ ", ""),
                    "sort_local": sort_local.replace("__device__ ", "")}
    d = tmp_path_factory.mktemp("nrlevels")
    cpp, so = d / "nrlevels.cpp", d / "nrlevels.so"
    cpp.write_text(src)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(so), str(cpp)],
                   check=True)
    lib = ctypes.CDLL(str(so))
    lib.nr_emulate.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int)]
    return lib


@pytest.mark.parametrize("n,kind", [(600, "random"), (2000, "ties"), (5000, "random"), (5000, "runs"),
                                    (20000, "ties"), (20000, "descending"), (65536, "random")])
def test_level_emulation_matches_oracle_indexx(emulate, n, kind):
    rng = np.random.default_rng(n + len(kind))
    if kind == "random":
        arr = rng.random(n)
    elif kind == "ties":
        arr = rng.integers(0, 16, n).astype(np.float64)
    elif kind == "runs":
        arr = np.repeat(rng.random(n // 5 + 1), 5)[:n].copy()
    else:
        arr = np.sort(rng.random(n))[::-1].copy()
    perm = np.empty(n, dtype=np.int32)
    levels = ctypes.c_int()
    rc = emulate.nr_emulate(n, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(levels))
    assert rc == 0
    assert levels.value >= 1
    np.testing.assert_array_equal(perm, O.indexx(arr))
