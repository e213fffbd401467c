"""Learned SGS model restated in numpy (the library's sgpu_set_sgs_mlp path).

TEST INFRASTRUCTURE ONLY: tests/ use it as the checker of the tensor-core MLP
kernel and of the stress the learned model feeds into the step.  The model has
no counterpart in the reference; the transforms around it follow the
reference's conventions (bla/les.f:140-400 for the velocity gradient on the
nx x nz grid, les.f:1560-1640 for the stress back in Fourier space).

MLP: x (10) -> tanh(W1 x + b1) (64) -> tanh(W2 h1 + b2) (64) -> W3 h2 + b3 (6),
weights, x, h1, h2 rounded to BF16 (round to nearest even), sums in float64
here (the device sums in FP32), tanh in float32.
"""
import numpy as np


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def init_weights(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    w = {
        "w1": rng.standard_normal((64, 10)) / np.sqrt(10.0),
        "b1": 0.1 * rng.standard_normal(64),
        "w2": rng.standard_normal((64, 64)) / 8.0,
        "b2": 0.1 * rng.standard_normal(64),
        "w3": scale * rng.standard_normal((6, 64)) / 8.0,
        "b3": 0.1 * scale * rng.standard_normal(6),
    }
    return {k: v.astype(np.float32) for k, v in w.items()}


def mlp_forward(x, w, s_out=1.0):
    """x: (n, 10) float32 features -> (n, 6)."""
    x = bf16(x).astype(np.float64)
    a1 = x @ bf16(w["w1"]).astype(np.float64).T
    h1 = np.tanh((a1.astype(np.float32) + w["b1"]).astype(np.float32))
    a2 = bf16(h1).astype(np.float64) @ bf16(w["w2"]).astype(np.float64).T
    h2 = np.tanh((a2.astype(np.float32) + w["b2"]).astype(np.float32))
    a3 = bf16(h2).astype(np.float64) @ bf16(w["w3"]).astype(np.float64).T
    return (np.float32(s_out) * (a3.astype(np.float32) + w["b3"])).astype(np.float32)


def _to_phys(f, nx, nz):
    """Spectral (nz, nyp, nx/2) -> physical (nyp, nz, nx): the unnormalised
    synthesis of the reference (vcfftb then vrfftb), oddball kz dropped."""
    g = np.array(f, dtype=complex)
    g[nz // 2] = 0.0
    g = np.fft.ifft(g, axis=0) * nz                # z synthesis
    full = np.zeros((nz, g.shape[1], nx // 2 + 1), complex)
    full[:, :, :nx // 2] = g
    full[:, :, 0] = full[:, :, 0].real             # imaginary part of kx = 0 unused
    phys = np.fft.irfft(full, n=nx, axis=2) * nx   # x synthesis
    return np.transpose(phys, (1, 0, 2))


def _to_spec(p, nz):
    """Physical (nyp, nz, nx) -> spectral (nz, nyp, nx/2), unnormalised
    analysis (vrfftf then vcfftf), oddball zeroed."""
    nx = p.shape[2]
    s = np.fft.rfft(np.transpose(p, (1, 0, 2)), axis=2)[:, :, :nx // 2]
    s = np.fft.fft(s, axis=0)
    s[nz // 2] = 0.0
    return s


def velocity_gradient(u, v, w, ox, oz, alfa, beta, nx, nz):
    """du_i/dx_j (i-major) on the nx x nz grid, shape (9, nyp, nz, nx)."""
    a = alfa[None, None, :]
    b = beta[:, None, None]
    ia, ib = 1j * a, 1j * b
    spec = [ia * u, ia * v - oz, ib * u,
            ia * v, -(ia * u + ib * w), ib * v,
            ia * w, ox + ib * v, ib * w]
    return np.stack([_to_phys(f, nx, nz) for f in spec])


def learned_tau(state, alfa, beta, nx, nz, w, s_in, s_y, s_out):
    """Spectral SGS stress (6, nz, nyp, nx/2) of the state slots (u, v, w,
    omega_x, omega_z), normalised by 1/(nx nz) as les.f stores it."""
    u, v, ww, ox, oz = state[:5]
    nyp = u.shape[1]
    grad = velocity_gradient(u, v, ww, ox, oz, alfa, beta, nx, nz)
    eta = np.cos(np.pi * np.arange(nyp) / (nyp - 1))
    feats = np.empty((nyp, nz, nx, 10), np.float32)
    for k in range(9):
        feats[..., k] = np.float32(s_in) * grad[k].astype(np.float32)
    feats[..., 9] = (np.float32(s_y) * (1.0 - np.abs(eta))).astype(np.float32)[:, None, None]
    tau = mlp_forward(feats.reshape(-1, 10), w, s_out).reshape(nyp, nz, nx, 6).astype(np.float64)
    return np.stack([_to_spec(tau[..., c] / (nx * nz), nz) for c in range(6)])


def box_filter_sample(state, alfa, beta, nx, nz, f):
    """Training sample of the learned model (sgpu_box_filter_sample): top-hat
    averages over cells of f x f points of the nx x nz grid of u_i, of the
    gradients and of u_i u_j; returns features (nyp, nz/f, nx/f, 10) = the
    nine filtered gradients and 1 - |y|, targets (nyp, nz/f, nx/f, 6) =
    <u_i u_j> - <u_i><u_j> (11 12 13 22 23 33), float64."""
    u, v, ww, ox, oz = state[:5]
    nyp = u.shape[1]
    vel = np.stack([_to_phys(q, nx, nz) for q in (u, v, ww)])
    grad = velocity_gradient(u, v, ww, ox, oz, alfa, beta, nx, nz)

    def box(p):
        return p.reshape(p.shape[:-2] + (nz // f, f, nx // f, f)).mean(axis=(-3, -1))

    ub = box(vel)
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    tau = np.stack([box(vel[i] * vel[j]) - ub[i] * ub[j] for i, j in pairs])
    eta = np.cos(np.pi * np.arange(nyp) / (nyp - 1))
    feats = np.empty((nyp, nz // f, nx // f, 10))
    feats[..., :9] = np.moveaxis(box(grad), 0, -1)
    feats[..., 9] = (1.0 - np.abs(eta))[:, None, None]
    return feats, np.moveaxis(tau, 0, -1)


def viscosity_weights(nu_t, a=0.1, s_in=0.2):
    """Weights under which the network is, to O((a s_in du)^2), the linear
    eddy-viscosity stress tau_ij = -2 nu_t S_ij: layer 1 passes the nine
    gradient features through tanh at slope a (small arguments), layer 2 is
    the identity through tanh, layer 3 forms -nu_t (du_i/dx_j + du_j/dx_i)."""
    w1 = np.zeros((64, 10), np.float32)
    w2 = np.zeros((64, 64), np.float32)
    w3 = np.zeros((6, 64), np.float32)
    for k in range(9):
        w1[k, k] = a
        w2[k, k] = 1.0
    g = -nu_t / (a * s_in)          # h2_k ~ a s_in du_k
    pairs = [(0, 0), (1, 3), (2, 6), (4, 4), (5, 7), (8, 8)]   # 11 12 13 22 23 33
    for c, (p, q) in enumerate(pairs):
        w3[c, p] += g
        w3[c, q] += g
    z = np.zeros(64, np.float32)
    return {"w1": w1, "b1": z, "w2": w2, "b2": z.copy(), "w3": w3, "b3": np.zeros(6, np.float32)}


# ---------------------------------------------------------------------------
# Training (sgpu_sgs_mlp_train): FP64 restatement of the loss, its gradient
# and the Adam step, on the packed weights W1 [64][10], b1 [64], W2 [64][64],
# b2 [64], W3 [6][64], b3 [6].
# ---------------------------------------------------------------------------
MLP_SLICES = (("w1", 0, (64, 10)), ("b1", 640, (64,)), ("w2", 704, (64, 64)), ("b2", 4800, (64,)),
              ("w3", 4864, (6, 64)), ("b3", 5248, (6,)))
MLP_NPAR = 5254


def mlp_pack(w):
    """Weights dict (init_weights) -> packed vector (float32)."""
    return np.concatenate([np.asarray(w[k], np.float32).ravel() for k, _, _ in MLP_SLICES])


def mlp_unpack(p):
    return {k: np.asarray(p[o:o + int(np.prod(sh))], np.float64).reshape(sh) for k, o, sh in MLP_SLICES}


def mlp_loss_grad(p, x, t):
    """Loss sum (y - t)^2 / (6 n) of y = W3 tanh(W2 tanh(W1 x + b1) + b2) + b3
    (no BF16 rounding, no scales) and its gradient, packed, in float64."""
    w = mlp_unpack(p)
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    n = x.shape[0]
    h1 = np.tanh(x @ w["w1"].T + w["b1"])
    h2 = np.tanh(h1 @ w["w2"].T + w["b2"])
    y = h2 @ w["w3"].T + w["b3"]
    r = y - t
    loss = float((r * r).sum() / (6 * n))
    d3 = 2.0 * r / (6 * n)
    g2 = (d3 @ w["w3"]) * (1 - h2 * h2)
    g1 = (g2 @ w["w2"]) * (1 - h1 * h1)
    grad = {"w1": g1.T @ x, "b1": g1.sum(0), "w2": g2.T @ h1, "b2": g2.sum(0), "w3": d3.T @ h2, "b3": d3.sum(0)}
    return loss, np.concatenate([grad[k].ravel() for k, _, _ in MLP_SLICES])


def adam_step(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (step counts from 1), float64."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v

