"""The step-3 pencil algebra (compiled for the host from the same source the
CUDA kernels use) against the reference's own setmacrhs + trid (tau branch)
and dcheb, called from the translated reference.  CPU only; the results
must be bit-identical because both evaluate the same operations in the
same order without fused multiply-add."""
import ctypes

import numpy as np
import pytest

from simson_b200 import build as sbuild

dp = ctypes.POINTER(ctypes.c_double)


def P(a):
    return a.ctypes.data_as(dp)


def I(v):
    return ctypes.byref(ctypes.c_int(v))


@pytest.fixture(scope="module")
def libs(request):
    from conftest import reference_available
    if not reference_available(16, 17, 16):
        pytest.skip("reference oracle unavailable")
    from build_ref import build
    ref = ctypes.CDLL(build(16, 17, 16))
    host = ctypes.CDLL(sbuild.build_hostcheck())
    host.sbh_tau_solve.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp]
    host.sbh_cheb_deriv.argtypes = [dp, dp, ctypes.c_int]
    return ref, host


def ref_tau(ref, lam, f, bc1, bc2):
    m, n = f.shape
    c = np.zeros(n); d = np.zeros(n); e = np.zeros(n); q = np.zeros(n + 2)
    x = np.zeros((m, n))
    hl = np.array([lam])
    fc = np.ascontiguousarray(f)
    ref.f_setmacrhs(P(x), P(fc), P(c), P(d), P(e), P(hl), I(1), I(n), I(m), I(1), I(n))
    bc = np.zeros((m, 2))
    bc[:, 0] = bc1
    bc[:, 1] = bc2
    xc = np.zeros((m, 2))
    ref.f_trid(P(x), P(xc), P(q), P(c), P(d), P(e), P(fc), P(bc), I(1), I(n), I(m), I(1), I(n), I(0))
    return x


@pytest.mark.parametrize("n", [17, 33, 65, 97, 129, 193])
@pytest.mark.parametrize("lam", [0.0, 3.7, 1.6e6, 6.3e6])
def test_tau_solver_bitwise(libs, n, lam):
    ref, host = libs
    rng = np.random.default_rng(n + int(lam))
    m = 5
    f = rng.standard_normal((m, n)) * np.exp(-0.1 * np.arange(n))
    bc1 = rng.standard_normal(m)
    bc2 = rng.standard_normal(m)
    xr = ref_tau(ref, lam, f, bc1, bc2)
    x = np.zeros((m, n))
    cp = np.zeros(n)
    wt = np.zeros(n)
    host.sbh_tau_solve(lam, n, m, P(np.ascontiguousarray(f)), P(x), P(bc1), P(bc2), P(cp), P(wt))
    assert np.array_equal(x, xr), np.abs(x - xr).max()


def test_tau_solver_zero_rhs_homogeneous(libs):
    """f = 0 with boundary rows (1, 1): the homogeneous solution phi_h used by
    the v/omega superposition (linearbl.f:505-512)."""
    ref, host = libs
    n, lam = 65, 2.4e6
    f = np.zeros((1, n))
    xr = ref_tau(ref, lam, f, np.array([1.0]), np.array([1.0]))
    x = np.zeros((1, n))
    cp, wt = np.zeros(n), np.zeros(n)
    host.sbh_tau_solve(lam, n, 1, P(f), P(x), P(np.array([1.0])), P(np.array([1.0])), P(cp), P(wt))
    assert np.array_equal(x, xr)
    # x(+1) = sum x_k = 2, x(-1) = sum (-1)^k x_k = 0
    assert abs(x.sum() - 2.0) < 1e-12 and abs((x * (-1.0) ** np.arange(n)).sum()) < 1e-12


@pytest.mark.parametrize("n", [17, 65, 193])
def test_cheb_deriv_bitwise(libs, n):
    ref, host = libs
    a = np.random.default_rng(n).standard_normal(n)
    b_ref = np.zeros(n)
    ref.f_dcheb(P(b_ref), P(a), I(n), I(1), I(1))
    b = np.zeros(n)
    host.sbh_cheb_deriv(P(a), P(b), n)
    assert np.array_equal(b, b_ref)
    # and it is the derivative: compare with numpy's Chebyshev derivative
    np.testing.assert_allclose(b[:-1], np.polynomial.chebyshev.chebder(a), rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("n", [8, 9, 12, 18, 32, 72, 96, 128, 192, 240, 256, 288, 384, 576])
def test_fft_passes_match_numpy(n):
    """The radix-8/9/6/4/2/3/5 Stockham passes of every transform of the step
    (host build of the device source) against numpy's FFT, both signs."""
    host = ctypes.CDLL(sbuild.build_hostcheck())
    host.sbh_fft.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int]
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    inp = np.ascontiguousarray(np.stack([x.real, x.imag], -1).ravel())
    out = np.zeros(2 * n)
    for sign, ref in ((-1, np.fft.fft(x)), (1, np.fft.ifft(x) * n)):
        assert host.sbh_fft(n, P(inp), P(out), sign) > 0
        y = out[0::2] + 1j * out[1::2]
        assert np.abs(y - ref).max() <= 1e-15 * n * np.abs(ref).max()


@pytest.mark.parametrize("n", [17, 65, 193])
@pytest.mark.parametrize("lam", [0.0, 3.7, 1.6e6, 6.3e6])
def test_tau_solver_reordered_sums(libs, n, lam):
    """The mixed path's tau solve (boundary sums accumulated in the backward
    sweep, derivative parity sums from the solution) against the reference's
    setmacrhs + trid: the same solution up to the summation order, and the
    parity sums of D x equal to those of the reference's dcheb."""
    ref, host = libs
    host.sbh_tau_solve_fast.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp]
    rng = np.random.default_rng(7 * n + int(lam))
    m = 5
    f = rng.standard_normal((m, n)) * np.exp(-0.1 * np.arange(n))
    bc1 = rng.standard_normal(m)
    bc2 = rng.standard_normal(m)
    xr = ref_tau(ref, lam, f, bc1, bc2)
    x = np.zeros((m, n))
    cp = np.zeros(n)
    ds = np.zeros(2 * m)
    host.sbh_tau_solve_fast(lam, n, m, P(np.ascontiguousarray(f)), P(x), P(bc1), P(bc2), P(cp), P(ds))
    scale = np.abs(xr).max(axis=1, keepdims=True)
    assert np.all(np.abs(x - xr) <= 1e-9 * scale), (np.abs(x - xr) / scale).max()
    for q in range(m):
        d = np.zeros(n)
        ref.f_dcheb(P(d), P(np.ascontiguousarray(xr[q])), I(n), I(1), I(1))
        dsc = np.abs(d).sum()
        assert abs(ds[2 * q] - d[0::2].sum()) <= 1e-9 * dsc
        assert abs(ds[2 * q + 1] - d[1::2].sum()) <= 1e-9 * dsc


@pytest.mark.parametrize("n", [9, 12, 96, 192, 576])
@pytest.mark.parametrize("prec", [0, 1])
def test_fft_paired_columns_match_numpy(n, prec):
    """Four interleaved columns through the paired-column passes (the layout
    of the CTA tiles), FP64 and FP32, both signs."""
    host = ctypes.CDLL(sbuild.build_hostcheck())
    host.sbh_fft4.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int]
    rng = np.random.default_rng(n + 7 * prec)
    x = rng.standard_normal((n, 4)) + 1j * rng.standard_normal((n, 4))
    inp = np.ascontiguousarray(np.stack([x.real, x.imag], -1).ravel())
    out = np.zeros(2 * 4 * n)
    tol = (1e-15 if prec == 0 else 2e-6) * n
    for sign, ref in ((-1, np.fft.fft(x, axis=0)), (1, np.fft.ifft(x, axis=0) * n)):
        assert host.sbh_fft4(n, P(inp), P(out), sign, prec) > 0
        y = (out[0::2] + 1j * out[1::2]).reshape(n, 4)
        assert np.abs(y - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("n", [72, 96, 240, 288, 576])
@pytest.mark.parametrize("prec", [0, 1])
def test_fixed_length_fft(n, prec):
    """The compile-time plans of the production transform lengths over 3, 4
    and 6 interleaved columns against numpy, both signs; with 4 columns they
    equal the runtime plan bit for bit (same passes, twiddles, butterflies)."""
    host = ctypes.CDLL(sbuild.build_hostcheck())
    host.sbh_cfft.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int]
    host.sbh_fft4.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int]
    tol = (1e-15 if prec == 0 else 2e-6) * n
    for cols in (3, 4, 6):
        rng = np.random.default_rng(n + 7 * prec + 100 * cols)
        x = rng.standard_normal((n, cols)) + 1j * rng.standard_normal((n, cols))
        inp = np.ascontiguousarray(np.stack([x.real, x.imag], -1).ravel())
        out = np.zeros(2 * cols * n)
        for sign, ref in ((-1, np.fft.fft(x, axis=0)), (1, np.fft.ifft(x, axis=0) * n)):
            assert host.sbh_cfft(n, cols, P(inp), P(out), sign, prec) > 0
            y = (out[0::2] + 1j * out[1::2]).reshape(n, cols)
            assert np.abs(y - ref).max() <= tol * np.abs(ref).max()
            if cols == 4:
                out4 = np.zeros_like(out)
                assert host.sbh_fft4(n, P(inp), P(out4), sign, prec) > 0
                assert np.array_equal(out, out4)


@pytest.mark.parametrize("n", [17, 33, 65, 97, 129, 193, 223])
def test_tensor_core_chebyshev_matrix(n):
    """The mixed path's tensor-core Chebyshev transforms, emulated in FP64 from
    their matrix image (even/odd folding, the two half matrices decoded from
    the tile layout as hi + lo, unfolding): every image entry is a TF32 value,
    forward and inverse equal the dense DCT-I of the reference's conventions
    to ~2^-21, and inverse after forward is the identity."""
    host = ctypes.CDLL(sbuild.build_hostcheck())
    host.sbh_chb_apply.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, dp, dp]
    N = n - 1
    j = np.arange(n)
    cosm = np.cos(np.pi * np.outer(j, j) / N)
    w = np.where((j == 0) | (j == N), 1.0, 2.0)
    cb = np.where((j == 0) | (j == N), 2.0, 1.0)
    scale = 1.0 / 3.0
    exact = {0: scale * cosm * w[None, :] / (N * cb[:, None]), 1: cosm}
    ncol = 7
    rng = np.random.default_rng(n)
    u = rng.standard_normal((n, ncol))
    res = {}
    for inv, s in ((0, scale), (1, 1.0)):
        out = np.zeros((n, ncol))
        assert host.sbh_chb_apply(n, inv, s, ncol, P(np.ascontiguousarray(u)), P(out)) > 0
        ref = exact[inv] @ u
        assert np.abs(out - ref).max() <= 2.0 ** -20 * np.abs(ref).max()
        res[inv] = out
    a = res[0]
    back = np.zeros((n, ncol))
    host.sbh_chb_apply(n, 1, 1.0, ncol, P(np.ascontiguousarray(a)), P(back))
    np.testing.assert_allclose(back, scale * u, atol=1e-5 * scale * np.abs(u).max())
