"""The shared-memory segment sort of the NR index sort emulation, on the CPU.

`nr_sort_local` in csrc/fsb_locmin.cu finishes every quicksort segment of
8..512 elements in one warp (k_nr_medium).  It is plain C++ apart from its
`__device__` qualifier, so this test compiles the function from the CUDA
source for the host with g++ and checks that, applied to a whole array of up
to 512 elements (what the GPU does for such an array), it gives exactly the
oracle's loc_min_3_indexx permutation (LocalMinima.f90:947-1046), ties
included.  Larger arrays reach it through the level-synchronous partition,
whose segments are independent, so the same equality holds per segment.
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


def _function_source(text, signature):
    start = text.index(signature)
    end = text.index("\n}\n", start) + 3  # the function's closing brace at column 0
    return text[start:end].replace("__device__ ", "")


@pytest.fixture(scope="module")
def sort_local(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    text = open(SRC).read()
    medium = int(text.split("constexpr int kNrMedium = ")[1].split(";")[0])
    body = _function_source(text, "__device__ bool nr_sort_local(")
    d = tmp_path_factory.mktemp("nrlocal")
    cpp, so = d / "nrlocal.cpp", d / "nrlocal.so"
    cpp.write_text("constexpr int kNrMedium = %d;\n%s\n"
                   'extern "C" int sort_local(double* k, int* i, int n) '
                   "{ return nr_sort_local(k, i, n) ? 0 : 1; }\n" % (medium, body))
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(so), str(cpp)],
                   check=True)
    lib = ctypes.CDLL(str(so))
    lib.sort_local.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    return lib, medium


def _arrays(rng, count, nmax):
    for t in range(count):
        n = int(rng.integers(1, nmax + 1))
        kind = t % 4
        if kind == 0:
            yield rng.random(n)
        elif kind == 1:
            yield rng.integers(0, 4, n).astype(np.float64)  # heavy ties
        elif kind == 2:
            yield np.sort(rng.random(n))[::-1].copy()  # descending
        else:
            yield np.repeat(rng.random((n + 2) // 3), 3)[:n].copy()  # runs of three equal keys


def test_segment_sort_matches_oracle_indexx(sort_local):
    lib, medium = sort_local
    rng = np.random.default_rng(2024)
    for arr in _arrays(rng, 1200, medium):
        key = arr.astype(np.float64).copy()
        ids = np.arange(arr.size, dtype=np.int32)
        rc = lib.sort_local(key.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), arr.size)
        assert rc == 0
        np.testing.assert_array_equal(ids, O.indexx(arr))
        np.testing.assert_array_equal(key, arr[ids])
