"""Seeded synthetic initial fields for the temporal channel.

The reference generates initial fields with a separate program (``bls``); the
channel workloads here use their own portable generator instead, so the same
field can be produced bit-for-bit in any language:

* base flow: laminar Poiseuille U(y) = 1 - y^2 on the Gauss-Lobatto points
  y_j = cos(pi j / (nyp-1)) (bla/preprbl.f:45);
* perturbation: complex Gaussian coefficients a, b (splitmix64 + Box-Muller)
  on the stored Fourier modes 0 <= kx <= kmax, |kz| <= kmax, except (0, 0);
  v = a (1-y^2)^2, omega_y = b (1-y^2)^2 and u, w from continuity exactly as
  the reference recovers them (bla/linearbl.f:1193-1212):
  u = i(alpha v' - beta omega_y)/k^2,  w = i(beta v' + alpha omega_y)/k^2.
  The kx = 0 column is made Hermitian (a(0,-kz) = conj a(0,kz)), so the field
  is real, divergence free and satisfies no-slip;
* scaling: the perturbation is scaled so that
  sqrt(<u'^2 + v'^2 + w'^2>/3) over the box equals ``rms`` (y integral with
  Clenshaw-Curtis weights, which integrate these polynomials exactly).

Arrays use the reference's main-storage layout: complex, shape
``(nz, nyp, nx//2)`` (kz index, y index, kx), kz index iz < nz/2 holds
kz = iz, iz > nz/2 holds kz = iz - nz, iz = nz/2 is the oddball mode (zero).
"""
from __future__ import annotations

import math

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014), the standard 64-bit mixer."""

    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        """Uniform in (0, 1]: 53 random bits."""
        return ((self.next() >> 11) + 1) * (1.0 / 9007199254740992.0)

    def normal_pair(self):
        u1, u2 = self.uniform(), self.uniform()
        r = math.sqrt(-2.0 * math.log(u1))
        return r * math.cos(2.0 * math.pi * u2), r * math.sin(2.0 * math.pi * u2)


def gl_points(nyp: int) -> np.ndarray:
    return np.cos(np.pi * np.arange(nyp) / (nyp - 1))


def cc_weights(nyp: int) -> np.ndarray:
    """Clenshaw-Curtis weights on the Gauss-Lobatto points for int_{-1}^{1}."""
    n = nyp - 1
    theta = np.pi * np.arange(nyp) / n
    w = np.zeros(nyp)
    for j in range(nyp):
        s = 0.0
        for k in range(1, n // 2 + 1):
            b = 1.0 if 2 * k == n else 2.0
            s += b * math.cos(2 * k * theta[j]) / (4 * k * k - 1)
        c = 1.0 if j in (0, n) else 2.0
        w[j] = c / n * (1.0 - s)
    return w


def wavenumbers(nx: int, nz: int, xl: float, zl: float):
    """alpha(kx index), beta(kz index) as bla/preprbl.f:36-43 defines them."""
    alfa = 2.0 * np.pi / xl * np.arange(nx // 2)
    beta = np.zeros(nz)
    for z in range(1, nz // 2 + 1):
        beta[z] = 2.0 * np.pi / zl * z
        beta[nz - z] = -2.0 * np.pi / zl * z
    return alfa, beta


def kz_index(kz: int, nz: int) -> int:
    return kz if kz >= 0 else nz + kz


def channel_field(nx: int, ny: int, nz: int, xl: float, zl: float, rms: float,
                  seed: int, kmax: int = 6, laminar: bool = True):
    """(u, v, w) complex arrays of shape (nz, ny, nx//2); see module doc."""
    nyp = ny
    y = gl_points(nyp)
    alfa, beta = wavenumbers(nx, nz, xl, zl)
    g = (1.0 - y * y) ** 2
    dg = -4.0 * y * (1.0 - y * y)
    shape = (nz, nyp, nx // 2)
    u = np.zeros(shape, complex)
    v = np.zeros(shape, complex)
    w = np.zeros(shape, complex)
    rng = SplitMix64(seed)
    kxm = min(kmax, nx // 2 - 1)
    kzm = min(kmax, nz // 2 - 1)
    coef = {}
    for kz in range(-kzm, kzm + 1):
        for kx in range(0, kxm + 1):
            ar, ai = rng.normal_pair()
            br, bi = rng.normal_pair()
            coef[(kx, kz)] = (complex(ar, ai), complex(br, bi))
    for (kx, kz), (a, b) in coef.items():
        if kx == 0 and kz == 0:
            continue
        if kx == 0 and kz < 0:
            a0, b0 = coef[(0, -kz)]
            a, b = a0.conjugate(), b0.conjugate()
        iz = kz_index(kz, nz)
        al, be = alfa[kx], beta[iz]
        k2 = al * al + be * be
        vv = a * g
        dv = a * dg
        om = b * g
        v[iz, :, kx] = vv
        u[iz, :, kx] = 1j * (al * dv - be * om) / k2
        w[iz, :, kx] = 1j * (be * dv + al * om) / k2
    if rms > 0:
        wy = cc_weights(nyp)
        e = 0.0
        for f in (u, v, w):
            m = np.abs(f) ** 2
            m[:, :, 1:] *= 2.0   # kx > 0 stands for +-kx
            e += float(np.einsum("zyx,y->", m, wy)) / 2.0
        scale = rms / math.sqrt(e / 3.0)
        u *= scale
        v *= scale
        w *= scale
    else:
        u[:] = 0
        v[:] = 0
        w[:] = 0
    if laminar:
        u[0, :, 0] += 1.0 - y * y
    return u, v, w
