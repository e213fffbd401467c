"""The bench workload itself, 384x193x384 (576x193x576 dealiased), checked
through properties that do not depend on an oracle run at this size (the
translated reference needs minutes per step here):

* laminar Poiseuille flow with constant flux is a fixed point of the step
  (the reference's own steady solution, bla/bla.f cflux branch), FP64 and
  mixed;
* the mixed path stays within the 1e-5 gate of the FP64 path after steps on
  the bench's seeded turbulent-like field;
* the state survives upload and download bit for bit (the reference layout
  of ur, ui at full size, 64-bit offsets).

These runs go through the compile-time FFT plans of length 576 and the
Chebyshev length 384 that the smaller parity grids do not reach."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

NX, NY, NZ, RE, XL, ZL, DT = 384, 193, 384, 9000.0, 2 * np.pi, np.pi, 0.002


def rel(a, b):
    """Relative L2 without the oddball plane kz = -nz/2 (left to the last
    nonlinear term by the reference and ignored by every reader)."""
    keep = np.ones(a.shape[0], bool)
    keep[a.shape[0] // 2] = False
    return float(np.linalg.norm(a[keep] - b[keep]) / np.linalg.norm(b[keep]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_laminar_fixed_point_at_bench_grid(precision):
    from simson_b200.bla import FP64, MIXED, Channel
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.0, 1)
    ch = Channel(NX, NY, NZ, RE, XL, ZL, DT, precision=FP64 if precision == "fp64" else MIXED)
    try:
        ch.set_velocity(u, v, w)
        ch.prhs()
        ch.step(3)
        s = ch.state(3)
        sc = ch.scalars()
    finally:
        ch.close()
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert np.abs(s[0] - u).max() <= tol * np.abs(u).max()
    assert np.abs(s[1]).max() <= tol and np.abs(s[2]).max() <= tol
    # constant flux: the pressure gradient of laminar flow, -2/Re
    assert abs(sc["px"] - (-2.0 / RE)) <= 1e-6 * 2.0 / RE


def test_mixed_vs_fp64_at_bench_grid():
    from simson_b200.bla import FP64, MIXED, Channel
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.1, 3)
    out = {}
    for prec in (FP64, MIXED):
        ch = Channel(NX, NY, NZ, RE, XL, ZL, DT, precision=prec)
        try:
            ch.set_velocity(u, v, w)
            ch.prhs()
            ch.step(5)
            out[prec] = ch.state(3)
        finally:
            ch.close()
    errs = [rel(out[MIXED][k], out[FP64][k]) for k in range(3)]
    assert max(errs) <= 1e-5, errs


def test_state_round_trip_at_bench_grid():
    from simson_b200.bla import FP64, Channel
    rng = np.random.default_rng(11)
    shape = (NZ, NY, NX // 2)
    slots = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(7)]
    ch = Channel(NX, NY, NZ, RE, XL, ZL, DT, precision=FP64)
    try:
        ch.set_state(slots)
        back = ch.state(7)
    finally:
        ch.close()
    for a, b in zip(back, slots):
        assert np.array_equal(a, b)
