"""The allocation-free diffusion entry point against the library's other paths.

fsb_diffusion_step_noalloc exists for callers that cannot call cudaMalloc
(real-time loops that must not stall on the allocator, frameworks that own all
device memory through their own pools): it runs the library's ADI diffusion
step on arrays the caller already owns, with its scratch in a static device
array.  Each case calls it through the C ABI twice in a row and checks both
results against a regular path on the same grid:

  * the step driver (fsb_execute_step) with erodibility kf = 0 and no uplift,
    so that the step changes the grid through diffusion only (boundary codes
    with at least one fixed side, which the full step needs);
  * the oracle's ADI step alone for the fully cyclic code 0000, which the full
    step refuses (depression routing needs a base level).

Cases cover every boundary kind (all fixed, x fixed, y fixed, fully cyclic),
kdsed off and on (with h above the basement on part of the grid, where the
sediment diffusivity applies) and the smallest grid, 3x3.
Tolerance: 1e-12 relative to max(|x|, 1), as in the other parity tests.
The file is collected last and passes alone or after the rest.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def bind(lib):
    f = lib.fsb_diffusion_step_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                  ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 6
    f.restype = ctypes.c_int
    return f


def grid(nx, ny, seed):
    rng = np.random.default_rng(seed)
    h0 = rng.random(nx * ny) * 50.0
    kd = rng.random(nx * ny) * 0.5 + 0.01
    b0 = h0.copy()
    b0[: (nx * ny) // 2] -= 2.0  # sediment cover on half of the grid
    return h0, b0, kd


class NoAlloc:
    """Device arrays of one grid and the entry point called on them."""

    def __init__(self, nx, ny, xl, yl, dt, bc, kdsed, h0, b0, kd):
        import torch
        import fastscapelib_fortran as fs
        self.f = bind(fs._lib)
        self.lib = fs._lib
        self.args = (nx, ny, xl, yl, dt, bc, kdsed)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.h = torch.tensor(h0, dtype=torch.float64, device=dev)
        self.b = torch.tensor(b0, dtype=torch.float64, device=dev)
        self.etot = torch.zeros_like(self.h)
        self.erate = torch.zeros_like(self.h)
        self.kd = torch.tensor(kd, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def call(self):
        import torch
        self.erate.zero_()  # the step driver's stream-power stage resets erate before diffusion
        torch.cuda.synchronize()
        rc = self.f(*self.args, self.kd.data_ptr(), self.h.data_ptr(), self.b.data_ptr(),
                    self.etot.data_ptr(), self.erate.data_ptr(),
                    ctypes.c_void_p(self.stream.cuda_stream))
        assert rc == 0, self.lib.fsb_last_error().decode()

    def fields(self):
        return {"h": self.h.cpu().numpy(), "basement": self.b.cpu().numpy(),
                "total_erosion": self.etot.cpu().numpy(), "erosion_rate": self.erate.cpu().numpy()}


@pytest.mark.parametrize("nx,ny,bc,kdsed", [(101, 83, 1010, -1.0), (101, 83, 1111, -1.0),
                                            (101, 83, 1111, 0.3), (64, 70, 101, -1.0),
                                            (64, 70, 101, 0.3), (3, 3, 1111, -1.0),
                                            (3, 3, 1010, 0.3)])
def test_noalloc_matches_step_driver(nx, ny, bc, kdsed):
    import fastscapelib_fortran as fs

    xl, yl, dt = 1.0e3 * (nx - 1), 1.0e3 * (ny - 1), 1.0e3
    h0, b0, kd = grid(nx, ny, nx * ny + bc)
    g = fs.FastScape()
    g.set_nx_ny(nx, ny)
    g.setup()
    g.set_xl_yl(xl, yl)
    g.set_dt(dt)
    g.init_h(h0)
    g.set_basement(b0)
    g.set_erosional_parameters(np.zeros(nx * ny), -1.0, 0.4, 1.0, kd, kdsed, 0.0, 0.0, -2.0)
    g.set_bc(bc)
    na = NoAlloc(nx, ny, xl, yl, dt, bc, kdsed, h0, b0, kd)
    for step in range(2):  # two calls in a row, each against the step driver
        na.call()
        g.execute_step()
        for name, got in na.fields().items():
            ref = np.empty(nx * ny)
            g.copy(name, ref)
            err = rel_err(got, ref)
            assert err <= TOL, (step, name, err)
    g.destroy()


@pytest.mark.parametrize("kdsed", [-1.0, 0.3])
def test_noalloc_fully_cyclic_matches_oracle(kdsed):
    import oracle as O

    nx, ny, bc = 40, 36, 0
    xl, yl, dt = 4.0e4, 3.5e4, 1.0e3
    h0, b0, kd = grid(nx, ny, 99)
    O.fastscape_init()
    O.fastscape_set_nx_ny(nx, ny)
    O.fastscape_setup()
    O.fastscape_set_xl_yl(xl, yl)
    O.fastscape_set_dt(dt)
    O.fastscape_init_h(h0.copy())
    O.fastscape_set_basement(b0)
    O.fastscape_set_erosional_parameters(np.zeros(nx * ny), -1.0, 0.4, 1.0, kd, kdsed, 0.0, 0.0,
                                         -2.0)
    O.fastscape_set_bc(bc)
    na = NoAlloc(nx, ny, xl, yl, dt, bc, kdsed, h0, b0, kd)
    for step in range(2):
        na.call()
        h_before = O.copy_double("h")
        O.diffusion_only()
        h_after = O.copy_double("h")
        got = na.fields()
        assert rel_err(got["h"], h_after) <= TOL, step
        assert rel_err(got["basement"], O.copy_double("basement")) <= TOL, step
        assert rel_err(got["total_erosion"], O.copy_double("total_erosion")) <= TOL, step
        assert rel_err(got["erosion_rate"], (h_before - h_after) / dt) <= TOL, step
    O.fastscape_destroy()


def test_noalloc_allocates_nothing_and_refuses_oversize():
    import torch

    nx, ny = 101, 83
    h0, b0, kd = grid(nx, ny, 1)
    na = NoAlloc(nx, ny, 1.0e5, 8.2e4, 1.0e3, 1010, -1.0, h0, b0, kd)
    na.call()
    dev = na.h.device
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    na.call()
    na.call()
    assert torch.cuda.mem_get_info(dev)[0] == free_before
    # sizes beyond the static scratch are refused with a clear message
    rc = na.f(300, 300, 1.0e5, 1.0e5, 1.0e3, 1010, -1.0, na.kd.data_ptr(), na.h.data_ptr(),
              na.b.data_ptr(), na.etot.data_ptr(), na.erate.data_ptr(),
              ctypes.c_void_p(na.stream.cuda_stream))
    assert rc != 0 and b"exceeds" in na.lib.fsb_last_error()
