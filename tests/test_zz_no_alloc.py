"""sgpu_nonlin_noalloc, the allocation-free nonlinear step for hosts that
cannot let the library call cudaMalloc, against sgpu_nonlin on the same
fields: two calls in a row, same tolerance as the step-2 parity tests.
Collected last so a failure here cannot hide the other tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_nonlin_noalloc_matches_sgpu_nonlin():
    import torch
    from simson_b200.bla import Channel, SgpuParams, load_library
    from simson_b200.fields import channel_field

    nx, ny, nz = 48, 65, 48
    xl, zl, re, dt = 4 * np.pi, 2 * np.pi, 4200.0, 0.01
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.05, 21)
    ch = Channel(nx, ny, nz, re, xl, zl, dt)
    ch.set_velocity(u, v, w)
    ch.prhs()
    fields = ch.state(5)  # u, v, w, omega_x, omega_z in the reference layout (nz, ny, nx/2)
    # caller-owned device buffers in the library's device layout (ny, nz, nx/2)
    dev_in = torch.from_numpy(np.ascontiguousarray(np.stack([f.transpose(1, 0, 2) for f in fields]))).cuda()
    out = torch.empty((3, ny, nz, nx // 2), dtype=torch.complex128, device="cuda")
    ch.nonlinbl()
    h_ref = [ch.get_slot(k) for k in (1, 2, 3)]
    cfl_ref = ch.scalars()["cfl"]

    lib = load_library()
    lib.sgpu_nonlin_noalloc.argtypes = [ctypes.POINTER(SgpuParams), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    prm = SgpuParams(nx, ny, nz, re, xl, zl, dt, 3, 1, 4.0 / 3.0, -2.0 / re, 0.0, 3, 0, 0)
    for call in range(2):
        out.fill_(float("nan"))
        cfl = ctypes.c_double(-1.0)
        rc = lib.sgpu_nonlin_noalloc(ctypes.byref(prm), ctypes.c_void_p(dev_in.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), ctypes.byref(cfl), None)
        torch.cuda.synchronize()
        assert rc == 0, rc
        h = out.cpu().numpy()
        for k in range(3):
            err = rel(h[k].transpose(1, 0, 2), h_ref[k])
            assert err < 1e-13, (call, k, err)
        assert abs(cfl.value * np.pi * dt - cfl_ref) <= 1e-12 * cfl_ref

    # beyond the static area: rejected without touching the GPU buffers
    big = SgpuParams(384, 193, 384, 9000.0, 2 * np.pi, np.pi, 0.002, 3, 1, 4.0 / 3.0, -2.0 / 9000.0, 0.0, 3, 0, 0)
    assert lib.sgpu_nonlin_noalloc(ctypes.byref(big), ctypes.c_void_p(dev_in.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), None, None) == -1
    ch.close()
