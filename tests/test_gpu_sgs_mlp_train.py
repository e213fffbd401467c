"""Training of the learned SGS model on the device (sgpu_sgs_mlp_train).

* Loss and gradient (FP32 on the device) against the FP64 restatement in
  oracle/sgs_mlp.py on 5000 random samples: each weight block within 1e-4
  relative L2, the loss within 1e-5; one Adam step against the update rule
  applied to the device's own gradient, within FP32 rounding; the gradient
  at the updated weights again within 1e-4.
* What training gains: samples from a resolved channel field box-filtered
  over 4 x 4 points (sgpu_box_filter_sample) split in halves; the network
  trained on one half predicts the deviatoric stress of the other half with
  a mean squared error below 0.8 of that of the eddy-viscosity model
  -2 C |S| S_ij with C fitted by least squares on the training half (the
  method without the network)."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

SLICES = ((0, 640), (640, 704), (704, 4800), (4800, 4864), (4864, 5248), (5248, 5254))


def test_gradient_and_adam_step_match_the_oracle():
    from sgs_mlp import adam_step, init_weights, mlp_loss_grad, mlp_pack
    from simson_b200.bla import Channel
    rng = np.random.default_rng(7)
    n = 5000
    x = rng.standard_normal((n, 10)).astype(np.float32)
    t = (0.3 * rng.standard_normal((n, 6))).astype(np.float32)
    p0 = mlp_pack(init_weights(2))
    z = np.zeros_like(p0)
    ch = Channel(16, 17, 16, 4200.0, 4 * np.pi, 2 * np.pi, 0.01)
    try:
        _, _, _, s0, loss0, g0 = ch.sgs_mlp_train(p0, z, z, 0, x, t, 0, 0.01)
        p1, m1, v1, s1, loss1, g1 = ch.sgs_mlp_train(p0, z, z, 0, x, t, 1, 0.01)
    finally:
        ch.close()
    assert s0 == 0 and s1 == 1
    lref, gref = mlp_loss_grad(p0.astype(np.float64), x, t)
    assert abs(loss0 - lref) <= 1e-5 * lref
    for a, b in SLICES:
        err = np.linalg.norm(g0[a:b] - gref[a:b]) / np.linalg.norm(gref[a:b])
        assert err <= 1e-4, (a, b, err)
    q1, qm, qv = adam_step(p0.astype(np.float64), 0.0, 0.0, g0.astype(np.float64), 1, 0.01)
    assert np.all(np.abs(p1 - q1) <= 1e-6 * np.abs(p0) + 1e-8)
    np.testing.assert_allclose(m1, qm, rtol=1e-6, atol=1e-30)
    np.testing.assert_allclose(v1, qv, rtol=1e-6, atol=1e-30)
    l1, g1ref = mlp_loss_grad(p1.astype(np.float64), x, t)
    assert abs(loss1 - l1) <= 1e-5 * l1
    for a, b in SLICES:
        assert np.linalg.norm(g1[a:b] - g1ref[a:b]) <= 1e-4 * np.linalg.norm(g1ref[a:b])


def _smagorinsky_basis(g):
    """-2 |S| S_ij (11 12 13 22 23 33) from the gradients g[..., 3 i + j]."""
    G = g.reshape(-1, 3, 3)
    S = 0.5 * (G + np.transpose(G, (0, 2, 1)))
    sabs = np.sqrt(2.0 * (S * S).sum(axis=(1, 2)))
    idx = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    return np.stack([-2.0 * sabs * S[:, i, j] for i, j in idx], axis=1)


def test_training_beats_the_eddy_viscosity_model():
    from sgs_mlp import init_weights, mlp_pack, mlp_unpack
    from simson_b200.bla import Channel
    nx, ny, nz = 96, 65, 96
    xl, zl = 2 * np.pi, np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 5, kmax=16)
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.002)
    try:
        ch.set_velocity(u, v, w)
        ch.prhs()
        ch.step(3)
        feats, tau = ch.box_filter_sample(4)
        feats = feats.reshape(-1, 10).astype(np.float64)
        tau = tau.reshape(-1, 6).astype(np.float64)
        tr = (tau[:, 0] + tau[:, 3] + tau[:, 5]) / 3.0
        dev = tau - tr[:, None] * np.array([1, 0, 0, 1, 0, 1.0])
        grads = feats[:, :9]
        s_in = 1.0 / grads.std()
        s_t = dev.std()
        x = np.concatenate([grads * s_in, feats[:, 9:]], axis=1)
        y = dev / s_t
        rng = np.random.default_rng(0)
        train = rng.random(x.shape[0]) < 0.5
        test = ~train
        # the method without the network: -2 C |S| S_ij, C by least squares
        m = _smagorinsky_basis(grads)
        c = (m[train] * dev[train]).sum() / (m[train] * m[train]).sum()
        mse_smag = float(((dev[test] - c * m[test]) ** 2).mean())
        p0 = mlp_pack(init_weights(0, scale=0.1))
        z = np.zeros_like(p0)
        _, _, _, _, loss_start, _ = ch.sgs_mlp_train(p0, z, z, 0, x[train], y[train], 0, 0.003)
        p, _, _, step, loss_end, _ = ch.sgs_mlp_train(p0, z, z, 0, x[train], y[train], 1500, 0.003)
    finally:
        ch.close()
    W = mlp_unpack(p)
    h1 = np.tanh(x[test] @ W["w1"].T + W["b1"])
    h2 = np.tanh(h1 @ W["w2"].T + W["b2"])
    pred = (h2 @ W["w3"].T + W["b3"]) * s_t
    mse_mlp = float(((dev[test] - pred) ** 2).mean())
    print("train loss %.3e -> %.3e; held-out MSE: network %.3e, eddy viscosity %.3e, no model %.3e"
          % (loss_start, loss_end, mse_mlp, mse_smag, float((dev[test] ** 2).mean())))
    assert step == 1500
    assert loss_end < 0.5 * loss_start
    assert mse_mlp < 0.8 * mse_smag
