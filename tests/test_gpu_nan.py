"""A non-finite value seeded in the host arrays before upload (the fault
injection of the reference-facing boundary, done on the host): the step runs
through it without a device fault, sgpu_get_scalars reports it -- SGPU_E_NAN
(the value reaches the kx = kz = 0 mode and px within one substep), or for
an infinite velocity already the CFL stop SGPU_E_CFL -- and the same context
steps normally again after a clean upload and prhs."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bad", [np.nan, np.inf])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_non_finite_state_is_reported(precision, bad):
    from simson_b200.bla import Channel, SimsonError
    nx, ny, nz = 48, 65, 48
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.05, 5)
    ub = np.array(u)
    ub[3, 20, 5] = bad
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=precision)
    try:
        ch.set_velocity(ub, v, w)
        ch.prhs()
        ch.step(1)
        with pytest.raises(SimsonError, match="non-finite" if np.isnan(bad) else "non-finite|CFL"):
            ch.scalars()
        ch.set_velocity(u, v, w)
        ch.prhs()
        ch.step(1)
        sc = ch.scalars()
        assert np.isfinite(sc["px"]) and np.isfinite(sc["cfl"])
    finally:
        ch.close()
