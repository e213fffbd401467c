"""The reference oracle (the reference's own Fortran, translated to C) against
known answers.  CPU only."""
import numpy as np
import pytest

from simson_b200.fields import cc_weights, channel_field, gl_points


def test_grid_and_weights(need_ref):
    need_ref(16, 17, 16)
    from refsim import RefSim
    r = RefSim(16, 17, 16, 4200.0, 4 * np.pi, 2 * np.pi, 0.01)
    eta, wint = r.grid()
    assert np.array_equal(eta, gl_points(17))
    np.testing.assert_allclose(wint, cc_weights(17), atol=1e-15)
    assert abs(wint.sum() - 2.0) < 1e-14


def test_laminar_poiseuille_is_fixed_point(need_ref):
    """U = 1 - y^2 with constant flux is a discrete steady state."""
    need_ref(16, 17, 16)
    from refsim import RefSim
    r = RefSim(16, 17, 16, 4200.0, 4 * np.pi, 2 * np.pi, 0.01)
    u, v, w = channel_field(16, 17, 16, 4 * np.pi, 2 * np.pi, 0.0, 1)
    r.set_velocity(u, v, w)
    r.start()
    r.step(10)
    assert np.abs(r.get_slot(1) - u).max() < 1e-12
    assert np.abs(r.get_slot(2)).max() < 1e-12
    s = r.scalars()
    assert abs(s["px"] + 2.0 / 4200.0) < 1e-12
    assert abs(s["t"] - 0.1) < 1e-12


def test_orr_sommerfeld_orszag_1971(need_ref):
    """A small Tollmien-Schlichting mode grows at Orszag's published rate:
    Re = 10000, alpha = 1, c = 0.23752649 + 0.00373967 i."""
    need_ref(4, 65, 4)
    from os_modes import least_stable_mode
    from refsim import RefSim
    n, re, alpha = 64, 10000.0, 1.0
    c, v, dv = least_stable_mode(n, re, alpha)
    assert abs(c - (0.23752649 + 0.00373967j)) < 1e-8
    r = RefSim(4, n + 1, 4, re, 2 * np.pi / alpha, 2 * np.pi, 0.01)
    eps = 1e-7
    U = np.zeros((4, n + 1, 2), complex)
    V = np.zeros_like(U)
    y = gl_points(n + 1)
    U[0, :, 0] = 1 - y * y
    V[0, :, 1] = eps * v
    U[0, :, 1] = 1j * eps * dv / alpha
    r.set_velocity(U, V, np.zeros_like(U))
    r.start()
    r.step(500)
    T = r.scalars()["t"]
    vt = r.get_slot(2)[0, :, 1]
    ratio = np.vdot(v, vt) / np.vdot(v, v) / eps
    c_meas = 1j * np.log(ratio) / (alpha * T)
    assert abs(c_meas.real - 0.23752649) < 2e-8
    assert abs(c_meas.imag - 0.00373967) < 2e-8
    pred = eps * v * np.exp(-1j * alpha * c * T)
    assert np.abs(vt - pred).max() / np.abs(pred).max() < 1e-7


def test_seeded_field_is_divergence_free_and_scaled():
    nx, ny, nz = 16, 17, 16
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.02, 7, laminar=False)
    from simson_b200.fields import wavenumbers
    from os_modes import cheb
    D, _ = cheb(ny - 1)
    alfa, beta = wavenumbers(nx, nz, xl, zl)
    div = 1j * alfa[None, None, :] * u + np.einsum("ij,zjx->zix", D, v) + 1j * beta[:, None, None] * w
    assert np.abs(div).max() < 1e-12
    wy = cc_weights(ny)
    e = 0.0
    for f in (u, v, w):
        m = np.abs(f) ** 2
        m[:, :, 1:] *= 2
        e += np.einsum("zyx,y->", m, wy) / 2
    assert abs(np.sqrt(e / 3) - 0.02) < 1e-14
    for f in (u, v, w):  # no-slip
        assert np.abs(f[:, 0, :]).max() < 1e-15 and np.abs(f[:, -1, :]).max() < 1e-15
    # Hermitian kx = 0 column
    for kz in range(1, 7):
        assert np.allclose(v[kz, :, 0], np.conj(v[nz - kz, :, 0]))


def test_amp_row_laminar_channel():
    """amp.stat row of the laminar Poiseuille profile U = 1 - y^2, no
    fluctuations: bulk Reynolds number (4/3) Re/2, wall shears Omega_z = 2y,
    h+ = sqrt(2 Re), 99 % thickness at the wall point, W bulk 0."""
    from amp_row import amp_row
    from simson_b200.fields import gl_points
    nyp, re = 33, 4200.0
    eta = gl_points(nyp)
    amp = np.zeros((20, nyp))
    amp[8] = 1 - eta ** 2
    amp[11] = 2 * eta
    row = amp_row(amp, 1.5, re, -2.0 / re)
    assert row[0] == 1.5 and np.all(row[1:9] == 0.0)
    assert abs(row[12] - 4.0 / 3.0 * re / 2) < 1e-10 * re
    assert row[13] == 2.0 and row[14] == -2.0
    assert abs(row[10] - np.sqrt(2 * re)) < 1e-12 * re
    assert row[15] == 2.0 and row[18] == 0.0
    # displacement thickness of 1 - y^2 over [-1, 1]: 2 - 4/3
    assert abs(row[16] - 2.0 / 3.0) < 1e-13


def test_bf16_rounding_of_the_mlp_oracle():
    from sgs_mlp import bf16
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0], np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1); 1 + 3 * 2^-8 -> 1 + 2^-6
    np.testing.assert_array_equal(bf16(x), np.array([1.0, 1.0, 1.0 + 2 ** -6, -2.5, 0.0], np.float32))


def test_pressure_of_mean_profiles_vanishes():
    """Pressure oracle (bla/nonlinp.f + bla/linearp.f, built with pressure =
    1): for any flow made of mean profiles U(y), W(y) the wall-normal
    nonlinear term is H2 = U U' + W W' = dE/dy, so p = phi - E is zero
    (up to roundoff) whatever the profiles; the pressure of a perturbed
    field is finite and not zero."""
    import os
    from build_ref import REF_BLA, lib_path
    if not (os.path.isdir(REF_BLA) or os.path.exists(lib_path(16, 17, 16, pressure=True))):
        pytest.skip("pressure oracle neither buildable nor prebuilt")
    from refsim import RefSim
    nx, ny, nz = 16, 17, 16
    xl, zl = 4 * np.pi, 2 * np.pi
    y = gl_points(ny)
    u = np.zeros((nz, ny, nx // 2), complex)
    w = np.zeros_like(u)
    u[0, :, 0] = (1 - y ** 2) * (1 + 0.3 * y)
    w[0, :, 0] = 0.2 * (1 - y ** 4)
    r = RefSim(nx, ny, nz, 4200.0, xl, zl, 0.01, pressure=True)
    r.set_velocity(u, np.zeros_like(u), w)
    r.start()
    p = r.pressure()
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    assert np.abs(p[keep]).max() < 1e-12
    uu, vv, ww = channel_field(nx, ny, nz, xl, zl, 0.05, 3)
    r.set_velocity(uu, vv, ww)
    r.start()
    p = r.pressure()
    assert np.isfinite(p).all() and np.abs(p[keep]).max() > 1e-6
