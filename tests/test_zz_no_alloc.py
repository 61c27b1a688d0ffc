"""The allocation-free diffusion entry point against the regular step driver.

fsb_diffusion_step_noalloc exists for callers that cannot call cudaMalloc
(host callbacks, real-time loops, frameworks that own all device memory): it
runs the library's ADI diffusion step on arrays the caller already owns, with
its scratch in a static device array.  This test calls it through the C ABI
twice in a row and checks each result against the regular entry point
(fsb_execute_step) run on the same grid with erodibility kf = 0 and no
uplift, so that the regular step changes the grid through diffusion only.
Tolerance: 1e-12 relative to max(|x|, 1), as in the other parity tests.
It lives in its own file, collected last, and passes alone or after the rest.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def test_noalloc_diffusion_matches_step_driver():
    import torch
    import fastscapelib_fortran as fs

    lib = fs._lib
    lib.fsb_diffusion_step_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                               ctypes.c_double] + [ctypes.c_void_p] * 6
    lib.fsb_diffusion_step_noalloc.restype = ctypes.c_int

    nx, ny, xl, yl, dt, bc = 101, 83, 1.0e5, 8.2e4, 1.0e3, 1010
    rng = np.random.default_rng(7)
    h0 = rng.random(nx * ny) * 50.0
    kd = rng.random(nx * ny) * 0.5 + 0.01

    # regular entry point: the step driver with no erosion and no uplift
    g = fs.FastScape()
    g.set_nx_ny(nx, ny)
    g.setup()
    g.set_xl_yl(xl, yl)
    g.set_dt(dt)
    g.init_h(h0)
    g.set_erosional_parameters(np.zeros(nx * ny), -1.0, 0.4, 1.0, kd, -1.0, 0.0, 0.0, -2.0)
    g.set_bc(bc)

    dev = torch.device("cuda", torch.cuda.current_device())
    h = torch.tensor(h0, dtype=torch.float64, device=dev)
    b = h.clone()
    etot = torch.zeros_like(h)
    erate = torch.zeros_like(h)
    kd_d = torch.tensor(kd, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def call():
        erate.zero_()  # the step driver's stream-power stage resets erate before diffusion
        torch.cuda.synchronize()
        rc = lib.fsb_diffusion_step_noalloc(nx, ny, xl, yl, dt, bc, -1.0, kd_d.data_ptr(),
                                            h.data_ptr(), b.data_ptr(), etot.data_ptr(),
                                            erate.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.fsb_last_error().decode()

    call()  # the first call on a device resolves the static array's address
    g.execute_step()
    for step in range(2):
        if step:
            call()
            g.execute_step()
        for name, t in (("h", h), ("basement", b), ("total_erosion", etot),
                        ("erosion_rate", erate)):
            ref = np.empty(nx * ny)
            g.copy(name, ref)
            err = rel_err(t.cpu().numpy(), ref)
            assert err <= 1e-12, (step, name, err)
    # the calls themselves allocate no device memory
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    call()
    call()
    assert torch.cuda.mem_get_info(dev)[0] == free_before

    # sizes beyond the static scratch are refused with a clear message
    rc = lib.fsb_diffusion_step_noalloc(300, 300, xl, yl, dt, bc, -1.0, kd_d.data_ptr(),
                                        h.data_ptr(), b.data_ptr(), etot.data_ptr(),
                                        erate.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
    assert rc != 0 and b"exceeds" in lib.fsb_last_error()
    g.destroy()
