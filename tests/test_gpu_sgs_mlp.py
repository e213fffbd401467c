"""Learned SGS model (no reference counterpart): the tensor-core MLP kernel
against the numpy restatement in oracle/sgs_mlp.py, and the stress it feeds
into the step against the same restatement applied to the state (velocity
gradient on the nx x nz grid, MLP, transform back).

Tolerance: weights and activations are BF16, so a sum that the device
accumulates in a different FP32 order can round an activation to the
neighbouring BF16 value; outputs agree within 1e-3 relative L2 (typically
~1e-6) and 1e-2 of the largest output in any single value."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


def _close(got, want, rel_l2=1e-3, rel_max=1e-2):
    err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)
    mx = np.abs(got - want).max() / max(np.abs(want).max(), 1e-30)
    assert err < rel_l2 and mx < rel_max, (err, mx)
    return err


@pytest.mark.parametrize("n", [1, 127, 384, 5000])
def test_mlp_kernel_matches_numpy(n):
    from sgs_mlp import init_weights, mlp_forward
    from simson_b200.bla import Channel
    w = init_weights(3)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, 10)).astype(np.float32)
    ch = Channel(16, 17, 16, 4200.0, 2 * np.pi, np.pi, 0.005)
    y = ch.sgs_mlp_eval(w, x, s_out=0.5)
    ch.close()
    _close(y, mlp_forward(x, w, s_out=0.5))


def test_mlp_kernel_two_calls_and_weight_change():
    from sgs_mlp import init_weights, mlp_forward
    from simson_b200.bla import Channel
    rng = np.random.default_rng(1)
    x = rng.standard_normal((1000, 10)).astype(np.float32)
    ch = Channel(16, 17, 16, 4200.0, 2 * np.pi, np.pi, 0.005)
    for seed in (4, 5, 4):
        w = init_weights(seed)
        _close(ch.sgs_mlp_eval(w, x), mlp_forward(x, w))
    ch.close()


def test_learned_stress_matches_numpy():
    from sgs_mlp import init_weights, learned_tau
    from simson_b200.bla import Channel
    from simson_b200.fields import wavenumbers
    nx, ny, nz = 32, 33, 32
    xl, zl = 2 * np.pi, np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 12, kmax=14)
    weights = init_weights(7, scale=1e-3)
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005)
    ch.set_velocity(u, v, w)
    ch.start()
    ch.set_sgs_mlp(weights, s_in=0.5, s_y=2.0, s_out=1.0)
    start = ch.state(5)
    ch.substep()
    got = ch.sgs_stress()
    alfa, beta = wavenumbers(nx, nz, xl, zl)
    want = learned_tau(start, alfa, beta, nx, nz, weights, 0.5, 2.0, 1.0)
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    for c in range(6):
        _close(got[c][keep], want[c][keep])
    ch.close()


def test_learned_model_in_the_step():
    """64x97x64 (the LES configuration), 30 substeps with a network whose
    weights make it a linear eddy viscosity nu_t = 1e-5: the run stays
    finite, the model removes kinetic energy, and the mixed-precision path
    stays within 1e-5 of the FP64 one.  The stress is explicit in time, so a
    constant nu_t must stay below the diffusion limit of the wall-refined
    Chebyshev grid (about 1e-4 here; the eddy-viscosity model keeps nu_t small
    at the walls through Delta and C).  Random weights give a stress with no
    dissipative structure; such runs are not a precision test."""
    from sgs_mlp import viscosity_weights
    from simson_b200.bla import FP64, MIXED, Channel
    nx, ny, nz = 64, 97, 64
    xl, zl = 2 * np.pi, np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 4, kmax=30)
    weights = viscosity_weights(1e-5)
    out = {}
    for tag, prec, model in (("none", FP64, False), ("fp64", FP64, True), ("mixed", MIXED, True)):
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005, precision=prec)
        ch.set_velocity(u, v, w)
        ch.start()
        if model:
            ch.set_sgs_mlp(weights, s_in=0.2, s_y=1.0, s_out=1.0)
        ch.substeps(30)
        out[tag] = np.stack(ch.state(3))
        ch.close()
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    assert np.all(np.isfinite(out["fp64"]))
    energy = {k: float(np.sum(np.abs(v[:, keep, :, 1:]) ** 2)) for k, v in out.items()}
    assert energy["fp64"] < energy["none"], energy
    d_mixed = np.linalg.norm((out["mixed"] - out["fp64"])[:, keep]) / np.linalg.norm(out["fp64"][:, keep])
    assert d_mixed < 1e-5, d_mixed


def test_viscosity_network_is_an_eddy_viscosity():
    """The stress of the eddy-viscosity weights against -2 nu_t S_ij formed
    from the same velocity gradient (numpy), on the device path."""
    from sgs_mlp import learned_tau, viscosity_weights
    from simson_b200.bla import Channel
    from simson_b200.fields import wavenumbers
    nx, ny, nz = 32, 33, 32
    xl, zl = 2 * np.pi, np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 12, kmax=14)
    nu = 1e-4
    weights = viscosity_weights(nu)
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005)
    ch.set_velocity(u, v, w)
    ch.start()
    ch.set_sgs_mlp(weights, s_in=0.2, s_y=1.0, s_out=1.0)
    start = ch.state(5)
    ch.substep()
    got = ch.sgs_stress()
    ch.close()
    alfa, beta = wavenumbers(nx, nz, xl, zl)
    a, b = alfa[None, None, :], beta[:, None, None]
    uu, vv, ww, ox, oz = start
    ia, ib = 1j * a, 1j * b
    g = [ia * uu, ia * vv - oz, ib * uu, ia * vv, -(ia * uu + ib * ww), ib * vv, ia * ww, ox + ib * vv, ib * ww]
    pairs = [(0, 0), (1, 3), (2, 6), (4, 4), (5, 7), (8, 8)]
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    for c, (p, q) in enumerate(pairs):
        want = -nu * (g[p] + g[q])
        # tanh(a x) = a x (1 - (a x)^2 / 3 ...), BF16 weights and
        # activations (2^-9 relative each): within 3 %
        _close(got[c][keep], want[keep], rel_l2=3e-2, rel_max=5e-2)
