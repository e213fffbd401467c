"""sgpu_offload_steps (the driver keeps the state; every step uploads the 7
slots from its arrays and downloads the result into them, the copies of
consecutive steps pipelined in pieces of each slot, the first substep's step
2 started before p_v, p_omega have arrived) must equal the same steps done one by
one with sgpu_upload_state / sgpu_step_rk / sgpu_download_state, bit for
bit, FP64 and mixed."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spatial", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_offload_steps_equal_step_by_step(precision, spatial):
    """spatial: a spatially developing channel (fringe towards the Poiseuille
    base flow, no constant flux), whose step 2 also reads the fringe while
    the offload call starts it under the upload of p_v, p_omega."""
    from simson_b200.bla import Channel, PinnedArray, base_flow
    nx, ny, nz = 48, 65, 48
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.05, 9)
    shape = (7, nz, ny, nx // 2)
    out = []
    for mode in ("steps", "offload"):
        if spatial:
            ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, cflux=False, px=0.0, precision=precision)
            ch.set_base_flow(*base_flow(4, ny, 3 * nx // 2))
            ch.set_fringe(fstart=-4.0, fend=0.0, frise=2.0, ffall=1.0, fmax=1.0)
        else:
            ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=precision)
        hr, hi = PinnedArray(shape), PinnedArray(shape)
        try:
            ch.set_velocity(u, v, w)
            ch.prhs()
            ch.download_raw(hr.ptr, hi.ptr, 7)
            if mode == "steps":
                for _ in range(3):
                    ch.upload_raw(hr.ptr, hi.ptr, 7)
                    ch.step(1)
                    ch.download_raw(hr.ptr, hi.ptr, 7)
            else:
                ch.offload_steps(hr.ptr, hi.ptr, 3)
            out.append((hr.array.copy(), hi.array.copy(), ch.scalars()["px"]))
        finally:
            hr.free()
            hi.free()
            ch.close()
    (r0, i0, p0), (r1, i1, p1) = out
    assert np.array_equal(r0, r1) and np.array_equal(i0, i1)
    assert p0 == p1
