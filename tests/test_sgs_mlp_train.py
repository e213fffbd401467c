"""The FP64 restatement of the learned model's training (oracle/sgs_mlp.py)
on the CPU: its gradient against central finite differences of its loss,
and the Adam update against the published update rule written out."""
import numpy as np

from sgs_mlp import MLP_NPAR, adam_step, init_weights, mlp_loss_grad, mlp_pack


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = mlp_pack(init_weights(1)).astype(np.float64)
    x = rng.standard_normal((7, 10))
    t = rng.standard_normal((7, 6))
    loss, g = mlp_loss_grad(p, x, t)
    assert g.shape == (MLP_NPAR,) and loss > 0
    h = 1e-6
    for e in rng.choice(MLP_NPAR, 60, replace=False).tolist() + [0, 639, 640, 703, 704, 4799, 4800, 4863, 4864,
                                                                 5247, 5248, 5253]:
        q = p.copy()
        q[e] += h
        lp, _ = mlp_loss_grad(q, x, t)
        q[e] -= 2 * h
        lm, _ = mlp_loss_grad(q, x, t)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[e]) <= 1e-7 * max(1.0, abs(g[e])) + 1e-9, (e, fd, g[e])


def test_adam_step_rule():
    rng = np.random.default_rng(4)
    p, g = rng.standard_normal(20), rng.standard_normal(20)
    m, v = np.zeros(20), np.zeros(20)
    p1, m1, v1 = adam_step(p, m, v, g, 1, 0.01)
    # first step: m/(1-b1) = g, v/(1-b2) = g^2, so the update is lr g / (|g| + eps)
    np.testing.assert_allclose(p1, p - 0.01 * g / (np.abs(g) + 1e-8), rtol=1e-12, atol=1e-15)
    p2, _, _ = adam_step(p1, m1, v1, g, 2, 0.01)
    np.testing.assert_allclose(p2, p1 - 0.01 * g / (np.abs(g) + 1e-8), rtol=1e-10, atol=1e-14)
