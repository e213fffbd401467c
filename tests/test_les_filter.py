"""ADM-RT filters (CPU): the tables built by the library's host code
(les_filter.h, through the host build libsimson_hostcheck) against the
reference's init_filter and bla.f filter set-up (translated oracle), the
filtered columns against the reference's gur after its start-up prhs, and
properties of the filter that hold whatever the reference: low pass plus high
pass is the identity, the homogeneous transfer function is 1 at k = 0, 1/2
at the cut-off and 0 at the grid Nyquist number."""
import ctypes

import numpy as np
import pytest

from simson_b200.fields import channel_field

dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(dp)


@pytest.fixture(scope="module")
def host():
    from simson_b200.build import build_hostcheck
    lib = ctypes.CDLL(build_hostcheck())
    lib.sbh_les_filter.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_int] + [dp] * 5
    lib.sbh_les_hpf_column.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] + [ctypes.c_int] * 4 + [dp, dp]
    lib.sbh_les_yfilter.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, dp, dp]
    return lib


def _tables(host, ny, nx, nz, cutoff, iord):
    g1 = np.empty((ny, 5)); g2 = np.empty((ny, 5))
    sx = np.empty(nx // 2 + 1); sz = np.empty(nz // 2 + 1); lpf = np.empty((nz, nx // 2))
    assert host.sbh_les_filter(ny, nx, nz, cutoff, iord, _p(g1), _p(g2), _p(sx), _p(sz), _p(lpf)) == 0
    return g1, g2, sx, sz, lpf


@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_filter_tables_match_reference(grid, host, need_ref):
    from refsim import RefSim
    nx, ny, nz = grid
    need_ref(nx, ny, nz)
    ref = RefSim(nx, ny, nz, 4200.0, 4 * np.pi, 2 * np.pi, 0.01)
    ref.set_les()
    r1, r2, _, rx, rz, rl = ref.filter_tables()
    g1, g2, sx, sz, lpf = _tables(host, ny, nx, nz, 1 / 1.5, 5)
    # closed forms in the reference, linear solves here: equal to rounding
    assert np.abs(g1.T - r1).max() < 1e-14
    assert np.abs(g2.T - r2).max() < 1e-14
    assert np.abs(sx - rx[:nx // 2 + 1]).max() < 1e-14
    assert np.abs(sz - rz[:nz // 2 + 1]).max() < 1e-14
    assert np.abs(lpf - rl).max() < 1e-14


@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_secondary_filter_tables_match_reference(grid, host, need_ref):
    """The dynamic HPF model's second filter (x/z transfer functions over a
    quarter of the wavenumbers, the same wall-normal stencils) against the
    reference's set-up of bla/bla.f:1520-1545."""
    from refsim import RefSim
    nx, ny, nz = grid
    need_ref(nx, ny, nz)
    host.sbh_les_filter2.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_int] + [dp] * 4
    ref = RefSim(nx, ny, nz, 4200.0, 4 * np.pi, 2 * np.pi, 0.01)
    ref.set_les(iles=3, cs=0.0)
    r1, r2, _, rl, rf = ref.filter2_tables()
    p1, p2 = ref.filter_tables()[:2]
    assert np.array_equal(r1, p1) and np.array_equal(r2, p2)  # the wall-normal filter is the primary's
    g1 = np.empty((ny, 5)); g2 = np.empty((ny, 5))
    lpf = np.empty((nz, nx // 2)); filt = np.empty((nz, nx // 2))
    assert host.sbh_les_filter2(ny, nx, nz, 1 / 1.5, 5, _p(g1), _p(g2), _p(lpf), _p(filt)) == 0
    assert np.abs(g1.T - r1).max() < 1e-14 and np.abs(g2.T - r2).max() < 1e-14
    assert np.abs(filt - rf).max() < 1e-14
    assert np.abs(lpf - rl).max() < 1e-14
    assert filt[0, nx // 4 + 1:].max() == 0.0  # nothing passes above kx = nx/4


@pytest.mark.parametrize("mode", [2, 1, 0])
def test_filtered_columns_match_reference(mode, host, need_ref):
    """The column routine the kernel runs, on the host, against the
    reference's gur after prhs (all three velocity components)."""
    from refsim import RefSim
    nx, ny, nz = 16, 17, 16
    need_ref(nx, ny, nz)
    u, v, w = channel_field(nx, ny, nz, 4 * np.pi, 2 * np.pi, 0.05, 3)
    ref = RefSim(nx, ny, nz, 4200.0, 4 * np.pi, 2 * np.pi, 0.01)
    ref.set_les(ihighorder=mode)
    ref.set_velocity(u, v, w)
    ref.start()
    for comp, f in ((1, u), (2, v), (3, w)):
        want = ref.gu(comp)
        got = np.empty_like(want)
        for iz in range(nz):
            for kx in range(nx // 2):
                col = np.ascontiguousarray(np.stack([f[iz, :, kx].real, f[iz, :, kx].imag], -1))
                out = np.empty((ny, 2))
                assert host.sbh_les_hpf_column(ny, nx, nz, 1 / 1.5, 5, mode, kx, iz, _p(col), _p(out)) == 0
                got[iz, :, kx] = out[:, 0] + 1j * out[:, 1]
        scale = np.abs(f).max()
        assert np.abs(got - want).max() <= 1e-13 * scale, (comp, np.abs(got - want).max())


def test_low_plus_high_is_identity(host):
    ny = 33
    rng = np.random.default_rng(5)
    d = rng.standard_normal(ny)
    lo = np.empty(ny); hi = np.empty(ny)
    assert host.sbh_les_yfilter(ny, 1 / 1.5, 0, _p(d), _p(lo)) == 0
    assert host.sbh_les_yfilter(ny, 1 / 1.5, 1, _p(d), _p(hi)) == 0
    np.testing.assert_allclose(lo + hi, d, rtol=0, atol=1e-13)
    # the walls are not filtered; constants and linear profiles pass the low pass
    assert lo[0] == d[0] and lo[-1] == d[-1]
    y = 1 + np.cos(np.pi * np.arange(ny) / (ny - 1))
    for prof in (np.ones(ny), y, y * y):
        out = np.empty(ny)
        host.sbh_les_yfilter(ny, 1 / 1.5, 0, _p(np.ascontiguousarray(prof)), _p(out))
        np.testing.assert_allclose(out, prof, rtol=0, atol=1e-12)


def test_homogeneous_transfer_function(host):
    """specx[i] = G(pi i / (nx/2)): 1 at 0, 1/2 at the cut-off pi/1.5 (the
    implicit filter is built for that), 0 at pi."""
    nx = 48  # nx/2 = 24: i = 16 is exactly the cut-off 2 pi/3
    _, _, sx, _, _ = _tables(host, 17, nx, 8, 1 / 1.5, 5)
    assert abs(sx[0] - 1) < 1e-15
    assert abs(sx[16] - 0.5) < 1e-14
    assert abs(sx[24]) < 1e-14
    assert np.all(np.diff(sx) <= 1e-15)
