"""Training samples of the learned SGS model (sgpu_box_filter_sample): the
top-hat box filter over f x f points of the nx x nz grid, the nine filtered
gradients, the wall distance and tau_ij = <u_i u_j> - <u_i><u_j>, against
the numpy restatement in oracle/sgs_mlp.py on the same (downloaded) state.
The device sums in FP64 and writes float32: each quantity within 2e-6 of its
largest magnitude, FP64 and mixed state storage, f = 3 and 4."""
import numpy as np
import pytest

from simson_b200.fields import channel_field, wavenumbers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("factor", [3, 4])
def test_box_filter_sample_matches_numpy(precision, factor):
    from sgs_mlp import box_filter_sample
    from simson_b200.bla import Channel
    nx, ny, nz = 48, 65, 48
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.05, 5)
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=precision)
    try:
        ch.set_velocity(u, v, w)
        ch.prhs()
        ch.step(2)
        feats, tau = ch.box_filter_sample(factor)
        state = ch.state(5)
    finally:
        ch.close()
    alfa, beta = wavenumbers(nx, nz, xl, zl)
    want_f, want_t = box_filter_sample(state, alfa, beta, nx, nz, factor)
    assert feats.shape == (ny, nz // factor, nx // factor, 10) and tau.shape == (ny, nz // factor, nx // factor, 6)
    for k in range(10):
        scale = np.abs(want_f[..., k]).max()
        assert np.abs(feats[..., k] - want_f[..., k]).max() <= 2e-6 * scale, ("feature", k)
    for c in range(6):
        scale = np.abs(want_t[..., c]).max()
        assert scale > 0.0
        assert np.abs(tau[..., c] - want_t[..., c]).max() <= 2e-6 * scale, ("tau", c)
    # a filter of one point leaves no subgrid stress
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=precision)
    try:
        ch.set_velocity(u, v, w)
        _, tau1 = ch.box_filter_sample(1)
    finally:
        ch.close()
    assert np.abs(tau1).max() <= 1e-7 * max(np.abs(want_t).max(), 1e-30) + 1e-12
