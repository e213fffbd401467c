"""ctypes wrapper around the translated reference ``bla`` (oracle/_ref).

TEST INFRASTRUCTURE ONLY: used by tests/, bench.py's CPU-baseline arm and
``__graft_entry__.smoke()`` as the checker; never by the product path.

Field layout at this interface is the reference's main storage,
``ur(memnx, memny, memnz, slot)`` (bla/par.f:111-120), seen from numpy as a
complex array of shape ``(nz, nyp, nx//2)`` per slot (kx fastest).  Slots:
1-3 u, v, w (Fourier x/z, physical y); 4-5 omega_x, omega_z; 6-7 the partial
right-hand sides p_v, p_omega_y (Chebyshev y).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _lib(nx, ny, nz, build=True, fma=False, pressure=False):
    import sys
    sys.path.insert(0, HERE)
    from build_ref import build as _build, lib_path
    path = (_build(nx, ny, nz, fma=fma, pressure=pressure) if build
            else lib_path(nx, ny, nz, fma=fma, pressure=pressure))
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.sref_setup.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int] * 3
    lib.sref_setup_rk.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int] * 4 + [ctypes.c_double] * 2
    lib.sref_set_slot.argtypes = [ctypes.c_int, dp, dp]
    lib.sref_get_slot.argtypes = [ctypes.c_int, dp, dp]
    lib.sref_scalars.argtypes = [dp]
    lib.sref_get_puw.argtypes = [dp]
    lib.sref_grid.argtypes = [dp, dp]
    lib.sref_dims.argtypes = [ctypes.POINTER(ctypes.c_int)]
    lib.sref_set_iamp.argtypes = [ctypes.c_int]
    lib.sref_set_les.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_int]
    lib.sref_get_tau.argtypes = [ctypes.c_int, dp, dp]
    lib.sref_get_filter.argtypes = [dp] * 6
    lib.sref_get_gu.argtypes = [ctypes.c_int, dp, dp]
    lib.sref_get_amp.argtypes = [dp]
    lib.sref_xys.argtypes = [ctypes.c_double, ctypes.c_int, dp, dp]
    lib.sref_pressure.argtypes = [dp, dp]
    lib.sref_get_filter2.argtypes = [dp] * 5
    lib.sref_set_spatial.argtypes = [ctypes.c_int] + [ctypes.c_double] * 5
    lib.sref_get_fringe.argtypes = [dp, dp]
    lib.sref_get_base.argtypes = [dp, dp]
    return lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class RefSim:
    """The reference channel time stepper (temporal channel, RK3/CN, cflux)."""

    def __init__(self, nx, ny, nz, re, xl, zl, dt, cflux=True, icfl=None, threads=1, build=True, fma=False,
                 pressure=False, nst=3, cflmaxin=0.8, tmax=0.0):
        """dt <= 0: the variable time step of bla.i (first step from getdt,
        then the CFL rule of bla/bla.f:2355-2380 with cflmax = cflmaxin
        sqrt(3) or sqrt(8)); nst: 3 or 4 RK stages."""
        self.lib = _lib(nx, ny, nz, build, fma, pressure)
        self.nst = nst
        if icfl is None:
            icfl = nst
        dims = (ctypes.c_int * 12)()
        self.lib.sref_dims(dims)
        self.dims = list(dims)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nyp = self.dims[4]
        if nst == 3 and dt > 0:
            self.lib.sref_setup(re, xl, zl, dt, int(cflux), int(icfl), int(threads))
        else:
            self.lib.sref_setup_rk(re, xl, zl, dt, int(cflux), int(icfl), int(threads), int(nst), float(cflmaxin),
                                   float(tmax))
        self.shape = (nz, self.nyp, nx // 2)

    def set_slot(self, slot, field):
        f = np.ascontiguousarray(field, dtype=np.complex128).reshape(self.shape)
        re_ = np.ascontiguousarray(f.real)
        im_ = np.ascontiguousarray(f.imag)
        self.lib.sref_set_slot(slot, _dp(re_), _dp(im_))

    def get_slot(self, slot):
        re_ = np.empty(self.shape)
        im_ = np.empty(self.shape)
        self.lib.sref_get_slot(slot, _dp(re_), _dp(im_))
        return re_ + 1j * im_

    def set_velocity(self, u, v, w):
        for k, f in enumerate((u, v, w), start=1):
            self.set_slot(k, f)

    def start(self):
        self.lib.sref_start()

    def substep(self):
        self.lib.sref_substep()

    def step(self, n=1):
        for _ in range(self.nst * n):
            self.lib.sref_substep()

    def nonlin_only(self):
        self.lib.sref_nonlin_only()

    def linear_only(self):
        self.lib.sref_linear_only()

    def scalars(self):
        s = np.empty(12)
        self.lib.sref_scalars(_dp(s))
        keys = ("px", "mflux", "t", "cfl", "an", "bn", "anp1", "bnp1", "cnp1", "it", "tc", "dtn")
        return dict(zip(keys, s))

    def puw(self):
        p = np.empty((2, self.ny))
        self.lib.sref_get_puw(_dp(p))
        return p

    def grid(self):
        eta = np.empty(self.nyp)
        wint = np.empty(self.nyp)
        self.lib.sref_grid(_dp(eta), _dp(wint))
        return eta, wint

    def set_les(self, cutoff_inv=1.5, iord=5, chi=0.2, ihighorder=2, iles=1, cs=0.0, ineg=1):
        """LES of sgs.i (bla/rparamles.f defaults): iles 1 ADM-RT, 2 eddy viscosity
        (cs = 0: dynamic Smagorinsky); filters set up as bla/bla.f:1489-1545."""
        self.lib.sref_set_les(int(iles), float(cutoff_inv), int(iord), float(chi), int(ihighorder),
                              float(cs), int(ineg))

    def set_spatial(self, fltype=4, fstart=-13.0, fend=0.0, frise=7.0, ffall=3.0, fmax=1.0):
        """Spatial simulation (spat = .true.) with the fringe of bla.i and the
        base flow of flow type fltype (4 Poiseuille, 5 Couette) computed by
        the reference's bflow; px = 0 and no constant flux follow at start()."""
        self.lib.sref_set_spatial(int(fltype), float(fstart), float(fend), float(frise), float(ffall), float(fmax))

    def fringe(self):
        """fring1, fring2 of bla/ffun.f (x pairs) at the current frame."""
        n = self.dims[3] // 2
        f1 = np.empty(n)
        f2 = np.empty(n)
        self.lib.sref_get_fringe(_dp(f1), _dp(f2))
        return f1, f2

    def base_flow(self):
        """bu1, bu2 of bla/bflow.f, shape (3, nyp, nxp/2+1) (the Fortran
        (nxp/2+1, nyp, 3) array)."""
        shape = (3, self.nyp, self.dims[3] // 2 + 1)
        b1 = np.empty(shape)
        b2 = np.empty(shape)
        self.lib.sref_get_base(_dp(b1), _dp(b2))
        return b1, b2

    def tau(self, comp):
        """SGS stress component comp (1..6 = 11 12 13 22 23 33), shape (nz, nyp, nx//2)."""
        re_ = np.empty(self.shape)
        im_ = np.empty(self.shape)
        self.lib.sref_get_tau(int(comp), _dp(re_), _dp(im_))
        return re_ + 1j * im_

    def filter_tables(self):
        """gewy1, gewy2, diags (5, nyp); gewspecx (nx/2+2); gewspecz (nz/2+2); lpfxz (nz, nx/2)."""
        nx, nz = self.dims[0], self.dims[2]
        g1 = np.empty((5, self.nyp)); g2 = np.empty((5, self.nyp)); dg = np.empty((5, self.nyp))
        sx = np.empty(nx // 2 + 2); sz = np.empty(nz // 2 + 2); lpf = np.empty((nz, nx // 2))
        self.lib.sref_get_filter(_dp(g1), _dp(g2), _dp(dg), _dp(sx), _dp(sz), _dp(lpf))
        return g1, g2, dg, sx, sz, lpf

    def filter2_tables(self):
        """The dynamic HPF model's secondary filter (bla/bla.f:1520-1545):
        gewy12, gewy22, diags2 as (5, nyp); lpfxz2, filtxz2 as (nz, nx/2)."""
        g1, g2, dg = (np.empty((5, self.nyp)) for _ in range(3))
        lpf = np.empty((self.nz, self.nx // 2))
        filt = np.empty((self.nz, self.nx // 2))
        self.lib.sref_get_filter2(_dp(g1), _dp(g2), _dp(dg), _dp(lpf), _dp(filt))
        return g1, g2, dg, lpf, filt

    def gu(self, comp):
        """High-pass filtered velocity component comp (1..3), shape (nz, nyp, nx//2)."""
        re_ = np.empty(self.shape)
        im_ = np.empty(self.shape)
        self.lib.sref_get_gu(int(comp), _dp(re_), _dp(im_))
        return re_ + 1j * im_

    def set_iamp(self, iamp):
        """Plane statistics (boxamp) every iamp substeps from the next step on."""
        self.lib.sref_set_iamp(int(iamp))

    def amp(self):
        """amp(nyp,20) as an array (20, nyp): amp[k-1, y-1] = amp(y, k)."""
        a = np.empty((20, self.nyp))
        self.lib.sref_get_amp(_dp(a))
        return a

    def xys(self, dtn, reset=False, nxys=96):
        """One statistics sample (bla/bla.f:2069-2107: boxxys on every plane
        with weight dtn) of the current state, added to the running sums
        (zeroed first with reset).  Returns (xys, sumw): xys[s-1, y, x] =
        xys(x+1, y+1, s) of the reference, shape (nxys, nyp, nx)."""
        out = np.empty((nxys, self.nyp, self.nx))
        sw = np.zeros(1)
        self.lib.sref_xys(float(dtn), 1 if reset else 0, _dp(out), _dp(sw))
        return out, float(sw[0])

    def pressure(self):
        """Pressure of the current state (bla/bla.f:2486-2527); needs
        pressure=True.  Complex (nz, nyp, nx/2), Fourier x/z, physical y."""
        re_ = np.empty(self.shape)
        im_ = np.empty(self.shape)
        if self.lib.sref_pressure(_dp(re_), _dp(im_)) != 0:
            raise RuntimeError("oracle built without pressure")
        return re_ + 1j * im_

    def state(self):
        return [self.get_slot(k) for k in range(1, 8)]
