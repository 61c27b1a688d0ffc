"""FastScape_VTK on the GPU: the files are byte-identical to the oracle's
(legacy binary VTK, big-endian float32, as the reference writes them with
-fconvert=big-endian) for the same surface, basement and field, with vex > 0
(topography only) and vex < 0 (topography, basement, sea level)."""
import os

import numpy as np
import pytest

import oracle as O
from fastscapelib_fortran import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("vex", [3.0, -2.0])
def test_vtk_files_match_the_oracle(tmp_path, vex):
    import fastscapelib_fortran as fs
    wl = W.mfd(37, 29, seed=91, nsteps=2)
    wl.apply(O)
    g = fs.FastScape()
    g.set_nx_ny(wl.nx, wl.ny)
    g.setup()
    g.set_xl_yl(wl.xl, wl.yl)
    g.set_dt(wl.dt)
    g.init_h(wl.h0.copy())
    g.set_erosional_parameters(wl.kf, wl.kfsed, wl.m, wl.n, wl.kd, wl.kdsed, wl.g1, wl.g2, wl.p)
    g.set_u(wl.u)
    g.set_bc(wl.bc)
    for _ in range(wl.nsteps):
        O.fastscape_execute_step()
        g.execute_step()
    g.set_h(O.copy_double("h"))  # the same surface on both sides
    g.set_basement(O.copy_double("basement"))
    f = O.copy_double("erosion_rate")
    (tmp_path / "gpu").mkdir()
    (tmp_path / "cpu").mkdir()
    g.vtk(f, vex, str(tmp_path / "gpu"))
    O.fastscape_vtk(f, vex, str(tmp_path / "cpu"))
    names = sorted(os.listdir(tmp_path / "cpu"))
    assert names == sorted(os.listdir(tmp_path / "gpu"))
    assert len(names) == (1 if vex > 0 else 3) and names[-1] == "Topography0000002.vtk"
    for n in names:
        assert (tmp_path / "gpu" / n).read_bytes() == (tmp_path / "cpu" / n).read_bytes(), n
    g.destroy()


def test_module_function_writes_to_vtk_dir(tmp_path, monkeypatch):
    import fastscapelib_fortran as fs
    monkeypatch.chdir(tmp_path)
    wl = W.plain_d8(21, 17, seed=92)
    wl.apply(fs)
    fs.fastscape_execute_step()
    fs.fastscape_vtk(np.zeros(wl.nn), np.array(1.0))
    assert (tmp_path / "VTK" / "Topography0000001.vtk").exists()
