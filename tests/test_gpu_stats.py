"""Plane statistics (the reference's boxamp, called by nonlinbl at the first
substep of a step when iamp > 0) and the amp.stat row (wampbl), computed by
sgpu_amplitudes, against the translated reference on the same state.

The per-plane sums run in a different order on the device (a parallel
reduction) than in the reference's serial loops, so on the same state they
agree to roundoff: each column within 1e-12 of its largest magnitude."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

COLS = [k for k in range(1, 21) if k != 13]   # amp(y,13) is never written by boxamp


def _pair(nx, ny, nz, rms, seed, need_ref):
    need_ref(nx, ny, nz)
    from refsim import RefSim
    from simson_b200.bla import Channel
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, rms, seed)
    ref = RefSim(nx, ny, nz, 4200.0, xl, zl, 0.01)
    ref.set_iamp(3)
    ref.set_velocity(u, v, w)
    ref.start()
    gpu = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01)
    gpu.set_velocity(u, v, w)
    gpu.start()
    return ref, gpu


def _check_amp(ga, ra, tol):
    for k in COLS:
        scale = np.abs(ra[k - 1]).max()
        err = np.abs(ga[k - 1] - ra[k - 1]).max()
        assert err <= tol * scale or (scale == 0.0 and err == 0.0), (k, err, scale)


@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_amplitudes_of_reference_state(grid, need_ref):
    """The statistics kernel alone: the reference's own state (after its
    partial right-hand side) uploaded, so only the summation order differs."""
    nx, ny, nz = grid
    ref, gpu = _pair(nx, ny, nz, 0.05, 7, need_ref)
    gpu.set_state(ref.state())
    amp, _ = gpu.amplitudes()
    ref.substep()
    _check_amp(amp, ref.amp(), 1e-12)


@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_amplitudes_match_reference(grid, need_ref):
    """End to end: the device's own start-up state, whose vorticity agrees
    with the reference's to ~1e-12, hence 1e-11 on the squared sums."""
    from amp_row import amp_row
    nx, ny, nz = grid
    ref, gpu = _pair(nx, ny, nz, 0.05, 7, need_ref)
    amp, row = gpu.amplitudes()
    # the reference evaluates boxamp on this state inside its first substep
    ref.substep()
    ra = ref.amp()
    _check_amp(amp, ra, 1e-11)
    want = amp_row(ra, 0.0, 4200.0, gpu.scalars()["px"])
    got = np.array([row[k] for k in gpu.AMP_ROW])
    np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-14)


def test_amplitudes_after_a_step(need_ref):
    """After one full step the statistics of the advanced state agree too
    (boxamp runs again at it = 4 with iamp = 3), to the 1e-10 to which the
    advanced vorticity fields agree (the mean Omega_z carries the
    ill-conditioned mass-flux correction of px)."""
    ref, gpu = _pair(16, 17, 16, 0.05, 9, need_ref)
    for _ in range(3):
        ref.substep()
        gpu.substep()
    amp, _ = gpu.amplitudes()
    ref.substep()
    _check_amp(amp, ref.amp(), 1e-10)


def test_amplitudes_mixed_close_to_fp64():
    """Mixed precision stores the fluctuations in FP32; its statistics stay
    within 1e-5 of the FP64 path's after ten steps."""
    from simson_b200.bla import FP64, MIXED, Channel
    nx, ny, nz = 48, 65, 48
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.02, 11)
    out = {}
    for prec in (FP64, MIXED):
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=prec)
        ch.set_velocity(u, v, w)
        ch.start()
        ch.substeps(30)
        out[prec] = ch.amplitudes()
        ch.close()
    a64, r64 = out[FP64]
    a32, r32 = out[MIXED]
    # the mean W and Omega_x stay near zero: compare them against max |U|
    for k in COLS:
        scale = np.abs(a64[k - 1]).max() if k not in (10, 11) else np.abs(a64[8]).max()
        assert np.abs(a32[k - 1] - a64[k - 1]).max() <= 1e-5 * scale, k
    for k in ("urms", "vrms", "wrms", "hplus", "re_bulk", "tau1", "tau2"):
        assert abs(r32[k] - r64[k]) <= 1e-5 * abs(r64[k]), (k, r32[k], r64[k])
