"""Per-plane fallback of the learned SGS model to the plain eddy-viscosity
model of bla/les.f (sgpu_set_sgs_fallback; no counterpart in the reference).

Each xz-plane sums P = tau_ij S_ij and |P| of the network's stress; a plane
whose sum P exceeds bound * sum |P| (predicted backscatter) takes the
dynamic Smagorinsky stress for that substep.  Checked:

* bound below -1 (every plane switches): the stress and the state equal the
  dynamic model's (sgpu_set_les iles = 2) bit for bit, the same kernels
  running on every plane;
* bound 1 (no plane switches): equal to the learned model without the
  fallback, bit for bit;
* bound 0: per plane, the stress is the dynamic model's on switched planes
  and the network's on the others; the plane sums agree with the numpy
  restatement (oracle/sgs_mlp.py: gradient, BF16 network) within the BF16
  tolerance of the network tests, and so do the switches wherever the sum is
  not within that tolerance of the bound."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

NX, NY, NZ, XL, ZL, RE, DT = 32, 33, 32, 2 * np.pi, np.pi, 4200.0, 0.005


def _channel(model, weights=None, bound=None):
    from simson_b200.bla import Channel
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.1, 12, kmax=14)
    ch = Channel(NX, NY, NZ, RE, XL, ZL, DT)
    ch.set_velocity(u, v, w)
    ch.start()
    if model == "dyn":
        ch.set_les(iles=2, cs=0.0, ineg=1)
    else:
        ch.set_sgs_mlp(weights, s_in=0.5, s_y=2.0, s_out=1.0)
        if bound is not None:
            ch.set_sgs_fallback(bound=bound, cs=0.0, ineg=1)
    return ch


def test_fallback_on_every_plane_is_the_dynamic_model():
    from sgs_mlp import init_weights
    a = _channel("mlp", init_weights(7, scale=1e-3), bound=-2.0)
    b = _channel("dyn")
    try:
        a.substep()
        b.substep()
        planes, _ = a.sgs_fallback_planes()
        assert planes.all()
        assert np.array_equal(a.sgs_stress(), b.sgs_stress())
        for _ in range(5):
            a.substep()
            b.substep()
        for k, (x, y) in enumerate(zip(a.state(5), b.state(5))):
            assert np.array_equal(x, y), k
    finally:
        a.close()
        b.close()


def test_fallback_on_no_plane_is_the_learned_model():
    from sgs_mlp import init_weights
    a = _channel("mlp", init_weights(7, scale=1e-3), bound=1.0)
    b = _channel("mlp", init_weights(7, scale=1e-3))
    try:
        for _ in range(3):
            a.substep()
            b.substep()
        planes, _ = a.sgs_fallback_planes()
        assert not planes.any()
        assert np.array_equal(a.sgs_stress(), b.sgs_stress())
        for x, y in zip(a.state(5), b.state(5)):
            assert np.array_equal(x, y)
    finally:
        a.close()
        b.close()


def _plane_sums(state, weights):
    """Restatement of the switch's plane sums: tau of the network (BF16, as
    the device rounds it) and S_ij of the resolved gradient on the nx x nz
    grid; returns sum P and sum |P| per plane."""
    from sgs_mlp import mlp_forward, velocity_gradient
    from simson_b200.fields import wavenumbers
    alfa, beta = wavenumbers(NX, NZ, XL, ZL)
    u, v, w, ox, oz = state[:5]
    g = velocity_gradient(u, v, w, ox, oz, alfa, beta, NX, NZ)  # (9, ny, nz, nx)
    eta = np.cos(np.pi * np.arange(NY) / (NY - 1))
    feats = np.empty((NY, NZ, NX, 10), np.float32)
    for k in range(9):
        feats[..., k] = np.float32(0.5) * g[k].astype(np.float32)
    feats[..., 9] = (np.float32(2.0) * (1.0 - np.abs(eta))).astype(np.float32)[:, None, None]
    tau = mlp_forward(feats.reshape(-1, 10), weights, 1.0).reshape(NY, NZ, NX, 6).astype(np.float64)
    s = [g[0], .5 * (g[1] + g[3]), .5 * (g[2] + g[6]), g[4], .5 * (g[5] + g[7]), g[8]]
    p = tau[..., 0] * s[0] + tau[..., 3] * s[3] + tau[..., 5] * s[5] + 2 * (
        tau[..., 1] * s[1] + tau[..., 2] * s[2] + tau[..., 4] * s[4])
    return p.sum(axis=(1, 2)), np.abs(p).sum(axis=(1, 2))


def test_fallback_by_plane():
    from sgs_mlp import init_weights
    weights = init_weights(2, scale=1e-3)
    a = _channel("mlp", weights, bound=0.0)
    b = _channel("mlp", weights)
    c = _channel("dyn")
    try:
        start = a.state(5)
        for ch in (a, b, c):
            ch.substep()
        planes, sums = a.sgs_fallback_planes()
        ta, tb, tc = a.sgs_stress(), b.sgs_stress(), c.sgs_stress()
    finally:
        for ch in (a, b, c):
            ch.close()
    p, pa = _plane_sums(start, weights)
    print("switched planes:", np.flatnonzero(planes).tolist())
    # the device's sums against the restatement (BF16 network)
    assert np.all(np.abs(sums[:, 0] - p) <= 2e-2 * pa + 1e-300), np.abs(sums[:, 0] - p) / pa
    assert np.all(np.abs(sums[:, 1] - pa) <= 2e-2 * pa + 1e-300)
    clear = np.abs(p) > 2e-2 * pa
    assert np.array_equal(planes[clear] == 1, (p > 0)[clear])
    assert 0 < planes.sum() < NY, planes  # this field and network give both kinds of plane
    # the stress is the dynamic model's on switched planes, the network's elsewhere
    for y in range(NY):
        want = tc[:, :, y] if planes[y] else tb[:, :, y]
        assert np.array_equal(ta[:, :, y], want), y
