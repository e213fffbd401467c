"""Python host side of the B200 channel step (ctypes over the C ABI).

The reference's interface for this path is the pair of plane-loop calls in the
``bla`` driver (``nonlinbl`` over xz-planes, ``linearbl`` over xy-planes,
bla/bla.f:2251-2290 and 2433-2476) plus the startup ``prhs`` (bla/bla.f:1562).
:class:`Channel` mirrors that driver for the temporal channel: the same
``bla.i`` parameters, the same main-storage layout and slot numbering, and the
same substep bookkeeping.  The state lives on the GPU; ``get_slot`` /
``set_slot`` copy it in the reference layout.

There is no CPU fallback: constructing a :class:`Channel` without the CUDA
library (or without a GPU) raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))

FP64 = 0
MIXED = 1


class SgpuParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("re", ctypes.c_double), ("xl", ctypes.c_double), ("zl", ctypes.c_double),
        ("dt", ctypes.c_double), ("nst", ctypes.c_int), ("cflux", ctypes.c_int),
        ("mflux", ctypes.c_double), ("px", ctypes.c_double), ("rot", ctypes.c_double),
        ("icfl", ctypes.c_int), ("precision", ctypes.c_int), ("device", ctypes.c_int),
    ]


class SgpuLesParams(ctypes.Structure):
    """sgs.i of the reference (bla/rparamles.f): iles 1 = ADM-RT, 2 = eddy viscosity."""
    _fields_ = [
        ("iles", ctypes.c_int), ("cutoff_inv", ctypes.c_double), ("iord", ctypes.c_int),
        ("chi", ctypes.c_double), ("ihighorder", ctypes.c_int),
        ("cs", ctypes.c_double), ("ineg", ctypes.c_int),
    ]


class SgpuSgsMlp(ctypes.Structure):
    _fields_ = [(n, ctypes.POINTER(ctypes.c_float)) for n in ("w1", "b1", "w2", "b2", "w3", "b3")] + [
        ("s_in", ctypes.c_float), ("s_y", ctypes.c_float), ("s_out", ctypes.c_float)]


class SgpuFringe(ctypes.Structure):
    """The fringe of bla.i (fstart, fend, frise, ffall, fmax) and the frame's x."""
    _fields_ = [("fstart", ctypes.c_double), ("fend", ctypes.c_double), ("frise", ctypes.c_double),
                ("ffall", ctypes.c_double), ("fmax", ctypes.c_double), ("xsc", ctypes.c_double)]


class SimsonError(RuntimeError):
    """A non-zero status of the C ABI; .code holds the SGPU_E_* value."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


_LIB = None


def load_library(build: bool = True):
    """Load (building if needed) ``simson_b200/_lib/libsimson_b200.so``."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.environ.get("SIMSON_LIB") or (_build.build() if build else _build.LIB)
    if not os.path.exists(path):
        raise SimsonError(f"CUDA library missing: {path}")
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    lib.sgpu_init.argtypes = [ctypes.POINTER(SgpuParams), ctypes.POINTER(vp)]
    lib.sgpu_finalize.argtypes = [vp]
    lib.sgpu_upload_state.argtypes = [vp, dp, dp, ctypes.c_int]
    lib.sgpu_download_state.argtypes = [vp, dp, dp, ctypes.c_int]
    lib.sgpu_upload_puw.argtypes = [vp, dp]
    lib.sgpu_download_puw.argtypes = [vp, dp]
    for fn in ("sgpu_prhs", "sgpu_nonlin", "sgpu_linear", "sgpu_sync"):
        getattr(lib, fn).argtypes = [vp]
    lib.sgpu_step_rk.argtypes = [vp, ctypes.c_int]
    lib.sgpu_get_scalars.argtypes = [vp, dp, ctypes.c_int]
    lib.sgpu_event_record.argtypes = [vp, ctypes.c_int]
    lib.sgpu_event_elapsed.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    lib.sgpu_launch_count.argtypes = [vp]
    lib.sgpu_launch_count.restype = ctypes.c_longlong
    lib.sgpu_error_string.restype = ctypes.c_char_p
    lib.sgpu_host_alloc.argtypes = [ctypes.c_ulonglong, ctypes.POINTER(vp)]
    lib.sgpu_host_free.argtypes = [vp]
    lib.sgpu_amplitudes.argtypes = [vp, dp, dp]
    lib.sgpu_xys_sample.argtypes = [vp, ctypes.c_double]
    lib.sgpu_xys_get.argtypes = [vp, dp, dp]
    lib.sgpu_xys_reset.argtypes = [vp]
    lib.sgpu_box_filter_sample.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_float)]
    lib.sgpu_pressure.argtypes = [vp, dp, dp]
    lib.sgpu_sgs_mlp_train.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                       ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                       ctypes.c_longlong, ctypes.c_int, ctypes.c_float,
                                       ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    lib.sgpu_set_les.argtypes = [vp, ctypes.POINTER(SgpuLesParams)]
    lib.sgpu_download_les.argtypes = [vp, dp, dp]
    lib.sgpu_download_sgs_stress.argtypes = [vp, dp, dp]
    fp = ctypes.POINTER(ctypes.c_float)
    lib.sgpu_set_sgs_mlp.argtypes = [vp, ctypes.POINTER(SgpuSgsMlp)]
    lib.sgpu_sgs_mlp_eval.argtypes = [vp, ctypes.POINTER(SgpuSgsMlp), fp, fp, ctypes.c_longlong]
    lib.sgpu_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.sgpu_set_wait_limit.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.sgpu_cfl_rate.argtypes = [vp, dp]
    lib.sgpu_set_dt.argtypes = [vp, ctypes.c_double]
    lib.sgpu_set_pencil_kernel.argtypes = [vp, ctypes.c_int]
    lib.sgpu_cfl_partial.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int)]
    lib.sgpu_cfl_set_global.argtypes = [vp, ctypes.c_double]
    lib.sgpu_set_sgs_fallback.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.sgpu_sgs_fallback_planes.argtypes = [vp, ctypes.POINTER(ctypes.c_int), dp]
    lib.sgpu_offload_steps.argtypes = [vp, dp, dp, ctypes.c_int]
    lib.sgpu_set_shard.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.sgpu_copy_block.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    lib.sgpu_fringe_function.argtypes = [ctypes.POINTER(SgpuFringe), ctypes.c_int, ctypes.c_double, dp]
    lib.sgpu_set_fringe.argtypes = [vp, ctypes.POINTER(SgpuFringe)]
    lib.sgpu_set_base_flow.argtypes = [vp, dp, dp]
    lib.sgpu_profile.argtypes = [vp, ctypes.c_int]
    lib.sgpu_profile_read.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    _LIB = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


SCALARS = ("px", "mflux", "t", "cfl", "an", "bn", "anp1", "bnp1", "cnp1", "it", "tc", "dt")


def fringe_function(nxp, xl, fstart, fend, frise, ffall, fmax, xsc=0.0):
    """The fringe function lambda at the nxp physical x points (bla/ffun.f;
    points 2k-2, 2k-1 are the reference's fring1(k), fring2(k)).  Host code of
    the library (sgpu_fringe_function); needs no GPU."""
    lib = load_library()
    lam = np.empty(nxp)
    f = SgpuFringe(fstart, fend, frise, ffall, fmax, xsc)
    rc = lib.sgpu_fringe_function(ctypes.byref(f), int(nxp), float(xl), _dp(lam))
    if rc != 0:
        raise SimsonError(f"sgpu_fringe_function: {lib.sgpu_error_string(rc).decode()} ({rc})", rc)
    return lam


def base_flow(fltype, nyp, nxp):
    """Base flow of a channel flow type as bla/cbflow.f:117-155 builds it:
    Poiseuille 1 - y^2 (fltype 1, 4) or Couette y (2, 5) in u, zero v and w,
    on the Gauss-Lobatto points y_j = cos(pi j/(nyp-1)).  Returns bu1, bu2 of
    shape (3, nyp, nxp/2+1) (the reference's (nxp/2+1, nyp, 3) array); the
    last x row is zero (bflow.f fills it with the periodic point)."""
    eta = np.cos(np.pi * np.arange(nyp) / (nyp - 1))
    if fltype in (1, 4):
        prof = 1.0 - eta ** 2
    elif fltype in (2, 5):
        prof = eta.copy()
    else:
        raise ValueError(f"flow type {fltype}: only the channel base flows (1, 2, 4, 5)")
    bu = np.zeros((3, nyp, nxp // 2 + 1))
    bu[0, :, :nxp // 2] = prof[:, None]
    return bu, bu.copy()


def base_flow_from_fields(u, v, w, nxp, nyp=None, u0low=0.0, w0low=0.0):
    """Base flow read from a velocity field, as bla/rbflow.f does for rbfl:
    the kz = 0 plane of u, v, w (complex (nz, nyp, nx/2), e.g. from
    simson_b200.ufile.read_u), the lower-wall values of u and w moved to
    u0low, w0low (rbflow.f:157-160), synthesised in x on the nxp-point grid
    (the spectrum zero-padded beyond nx/2; real part of kx = 0, as the real
    inverse transform of bla/cvecfft_acc.f takes it).  Returns bu1, bu2 as
    base_flow does."""
    fields = [np.asarray(q)[0] for q in (u, v, w)]  # (nyp, nx/2)
    nyp_f, nx2 = fields[0].shape
    if nyp is not None and nyp != nyp_f:
        raise ValueError("the base flow needs the field's y resolution (read it with varsiz)")
    spec = np.zeros((3, nyp_f, nxp // 2 + 1), np.complex128)
    for i, q in enumerate(fields):
        spec[i, :, :nx2] = q
    spec[0, :, 0] += u0low - spec[0, -1, 0].real
    spec[2, :, 0] += w0low - spec[2, -1, 0].real
    spec[:, :, 0] = spec[:, :, 0].real
    phys = np.fft.irfft(spec, n=nxp, axis=2) * nxp  # sum over +-kx, unnormalised
    bu1 = np.zeros((3, nyp_f, nxp // 2 + 1))
    bu2 = np.zeros_like(bu1)
    bu1[:, :, :nxp // 2] = phys[:, :, 0::2]
    bu2[:, :, :nxp // 2] = phys[:, :, 1::2]
    return bu1, bu2


class Channel:
    """Temporal channel (fltype=1, RK3/CN, tau, ibc=0) resident on one GPU."""

    def __init__(self, nx, ny, nz, re, xl, zl, dt, cflux=True, mflux=4.0 / 3.0, px=None,
                 rot=0.0, icfl=None, precision=FP64, device=0, nst=3):
        self.lib = load_library()
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dt = dt
        self.nst = nst
        if icfl is None:
            icfl = nst
        self.shape = (nz, ny, nx // 2)
        if px is None:
            px = -2.0 / re  # bla/bla.f:1630 first guess under cflux
        if isinstance(precision, str):
            precision = {"fp64": FP64, "mixed": MIXED}[precision.lower()]
        prm = SgpuParams(nx, ny, nz, re, xl, zl, dt, nst, int(cflux), mflux, px, rot, icfl, precision, device)
        self._ctx = ctypes.c_void_p()
        self._check(self.lib.sgpu_init(ctypes.byref(prm), ctypes.byref(self._ctx)), "sgpu_init")

    def _check(self, rc, what):
        if rc != 0:
            raise SimsonError(f"{what}: {self.lib.sgpu_error_string(rc).decode()} ({rc})", rc)

    def close(self):
        if getattr(self, "_ctx", None):
            self.lib.sgpu_finalize(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- state in the reference layout ---------------------------------
    def set_state(self, slots):
        """slots: list of complex arrays (nz, ny, nx//2) for slots 1..k."""
        k = len(slots)
        a = np.ascontiguousarray(np.stack([np.asarray(s, np.complex128).reshape(self.shape) for s in slots]))
        re_ = np.ascontiguousarray(a.real)
        im_ = np.ascontiguousarray(a.imag)
        self._check(self.lib.sgpu_upload_state(self._ctx, _dp(re_), _dp(im_), k), "upload")

    def set_velocity(self, u, v, w):
        self.set_state([u, v, w])

    def state(self, nslots=7):
        re_ = np.empty((nslots,) + self.shape)
        im_ = np.empty((nslots,) + self.shape)
        self._check(self.lib.sgpu_download_state(self._ctx, _dp(re_), _dp(im_), nslots), "download")
        return list(re_ + 1j * im_)

    def get_slot(self, slot):
        return self.state(slot)[slot - 1]

    def puw(self):
        p = np.empty((2, self.ny))
        self._check(self.lib.sgpu_download_puw(self._ctx, _dp(p)), "puw")
        return p

    def offload_steps(self, re_ptr, im_ptr, n):
        """n RK3 steps with the state round-tripped through the host arrays
        (all 7 slots, reference layout, pinned) every step, the copies of
        consecutive steps pipelined per slot (sgpu_offload_steps)."""
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.sgpu_offload_steps(self._ctx, ctypes.cast(re_ptr, dp), ctypes.cast(im_ptr, dp), n),
                    "offload_steps")

    # --- the reference's call sequence ----------------------------------
    def set_shard(self, ylo, yhi, zlo, zhi):
        """Compute only a shard of the domain: step 2 on the xz-planes
        ylo <= y < yhi, step 3 on the stored kz planes zlo <= iz < zhi
        (bla/par.f:102 z-slabs; simson_b200.shard moves the blocks)."""
        self._check(self.lib.sgpu_set_shard(self._ctx, ylo, yhi, zlo, zhi), "set_shard")

    def copy_block(self, slot0, nslots, ylo, yhi, zlo, zhi, buf_ptr=None, to_state=False, nosync=False):
        """Pack (to_state=False) or unpack a block of state slots between the
        state and the device buffer at buf_ptr ([slot][y][kz][kx], the
        state's storage); returns its size in bytes (buf_ptr None: size
        only).  nosync: only enqueue the copy on the library's stream."""
        n = ctypes.c_size_t(0)
        flag = int(to_state) | (2 if nosync else 0)
        self._check(self.lib.sgpu_copy_block(self._ctx, slot0, nslots, ylo, yhi, zlo, zhi,
                                             ctypes.c_void_p(buf_ptr) if buf_ptr else None, flag,
                                             ctypes.byref(n)), "copy_block")
        return n.value

    def set_pencil_kernel(self, warp=True):
        """Step 3 with one warp per pencil (True), one thread per pencil
        (False) or the automatic choice by grid size ("auto");
        sgpu_set_pencil_kernel."""
        self._check(self.lib.sgpu_set_pencil_kernel(self._ctx, 2 if warp == "auto" else int(bool(warp))),
                    "set_pencil_kernel")

    def set_wait_limit(self, limit=0, test_timeout=False):
        """Bounded waits of the tensor-core kernels: iterations per wait
        (0: default); test_timeout makes each launch's first wait run out
        (sgpu_set_wait_limit)."""
        self._check(self.lib.sgpu_set_wait_limit(self._ctx, int(limit), int(bool(test_timeout))), "set_wait_limit")

    def stream_ptr(self):
        """The library's CUDA stream (cudaStream_t) as an integer."""
        s = ctypes.c_void_p()
        self._check(self.lib.sgpu_stream(self._ctx, ctypes.byref(s)), "stream")
        return s.value or 0

    def cfl_partial(self):
        """(partial CFL maximum of this shard's planes, pending) -- see
        sgpu_cfl_partial."""
        m = ctypes.c_double()
        p = ctypes.c_int()
        self._check(self.lib.sgpu_cfl_partial(self._ctx, ctypes.byref(m), ctypes.byref(p)), "cfl_partial")
        return m.value, bool(p.value)

    def cfl_set_global(self, cflp):
        """The all-reduced partial maximum: the reference's stop test (raises
        SimsonError on CFL*dt > 10 or a non-finite value)."""
        self._check(self.lib.sgpu_cfl_set_global(self._ctx, float(cflp)), "cfl")

    def prhs(self):
        self._check(self.lib.sgpu_prhs(self._ctx), "prhs")

    start = prhs

    def nonlinbl(self):
        """Step 2 of the substep for all xz-planes (bla/nonlinbl.f)."""
        self._check(self.lib.sgpu_nonlin(self._ctx), "nonlin")

    def linearbl(self):
        """Step 3 of the substep for all xy-planes (bla/linearbl.f)."""
        self._check(self.lib.sgpu_linear(self._ctx), "linear")

    def substep(self):
        self.nonlinbl()
        self.linearbl()

    def step(self, n=1):
        """n full RK steps (nst substeps each), no host synchronisation."""
        self._check(self.lib.sgpu_step_rk(self._ctx, self.nst * n), "step")

    def cfl_rate(self):
        """CFL number per unit time step of the current state (bla/getdt.f)."""
        r = ctypes.c_double()
        self._check(self.lib.sgpu_cfl_rate(self._ctx, ctypes.byref(r)), "cfl_rate")
        return r.value

    def set_dt(self, dt):
        """Time step of the next full step (before prhs: of the first step)."""
        self.dt = dt
        self._check(self.lib.sgpu_set_dt(self._ctx, float(dt)), "set_dt")

    def substeps(self, n):
        self._check(self.lib.sgpu_step_rk(self._ctx, n), "step")

    def sync(self):
        self._check(self.lib.sgpu_sync(self._ctx), "sync")

    def scalars(self):
        s = np.empty(12)
        self._check(self.lib.sgpu_get_scalars(self._ctx, _dp(s), 12), "scalars")
        return dict(zip(SCALARS, s))

    def record(self, slot):
        self._check(self.lib.sgpu_event_record(self._ctx, slot), "event")

    def elapsed_ms(self, a, b):
        ms = ctypes.c_float()
        self._check(self.lib.sgpu_event_elapsed(self._ctx, a, b, ctypes.byref(ms)), "elapsed")
        return ms.value

    def upload_raw(self, re_ptr, im_ptr, nslots):
        """Upload from caller-owned host buffers (e.g. pinned), reference layout."""
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.sgpu_upload_state(self._ctx, ctypes.cast(re_ptr, dp), ctypes.cast(im_ptr, dp), nslots),
                    "upload")

    def download_raw(self, re_ptr, im_ptr, nslots):
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.sgpu_download_state(self._ctx, ctypes.cast(re_ptr, dp), ctypes.cast(im_ptr, dp), nslots),
                    "download")

    def pressure_raw(self, re_ptr, im_ptr):
        """sgpu_pressure into caller-owned host buffers (page-locked ones make
        the download run at full PCIe speed)."""
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.sgpu_pressure(self._ctx, ctypes.cast(re_ptr, dp), ctypes.cast(im_ptr, dp)), "pressure")

    def set_fringe(self, fstart, fend, frise, ffall, fmax, xsc=0.0):
        """Fringe forcing of a spatial run (bla/fring.f) from now on; fmax = 0
        turns it off."""
        f = SgpuFringe(fstart, fend, frise, ffall, fmax, xsc)
        self._check(self.lib.sgpu_set_fringe(self._ctx, ctypes.byref(f)), "set_fringe")

    def set_base_flow(self, bu1=None, bu2=None):
        """Base flow the fringe damps towards: bu1, bu2 of shape (3, nyp,
        nxp/2+1) as base_flow returns them; None: zero."""
        if bu1 is None:
            self._check(self.lib.sgpu_set_base_flow(self._ctx, None, None), "set_base_flow")
            return
        b1 = np.ascontiguousarray(bu1, np.float64)
        b2 = np.ascontiguousarray(bu2, np.float64)
        if b1.shape != b2.shape or b1.shape[0] != 3 or b1.shape[1] != self.ny:
            raise ValueError("base flow arrays of shape (3, nyp, nxp/2+1)")
        self._check(self.lib.sgpu_set_base_flow(self._ctx, _dp(b1), _dp(b2)), "set_base_flow")

    def set_les(self, cutoff_inv=1.5, iord=5, chi=0.2, ihighorder=2, iles=1, cs=0.0, ineg=1):
        """Large-eddy model (defaults of bla/rparamles.f): iles 1 ADM-RT, 2 eddy
        viscosity (cs = 0: dynamic Smagorinsky).  Call before prhs()."""
        p = SgpuLesParams(int(iles), float(cutoff_inv), int(iord), float(chi), int(ihighorder), float(cs),
                          int(ineg))
        self._check(self.lib.sgpu_set_les(self._ctx, ctypes.byref(p)), "set_les")

    def les_gu(self):
        """High-pass filtered velocities (gur, gui of the reference), shape (3, nz, ny, nx//2)."""
        shape = (3,) + self.shape
        re_ = np.empty(shape)
        im_ = np.empty(shape)
        self._check(self.lib.sgpu_download_les(self._ctx, _dp(re_), _dp(im_)), "download_les")
        return re_ + 1j * im_

    @staticmethod
    def _mlp_struct(weights, s_in, s_y, s_out):
        keep = {k: np.ascontiguousarray(weights[k], dtype=np.float32) for k in ("w1", "b1", "w2", "b2", "w3", "b3")}
        fp = ctypes.POINTER(ctypes.c_float)
        st = SgpuSgsMlp(*[keep[k].ctypes.data_as(fp) for k in ("w1", "b1", "w2", "b2", "w3", "b3")],
                        float(s_in), float(s_y), float(s_out))
        return st, keep

    def set_sgs_mlp(self, weights, s_in=1.0, s_y=1.0, s_out=1.0):
        """Learned SGS model: weights dict w1 (64,10), b1 (64), w2 (64,64), b2, w3 (6,64), b3 (6)."""
        st, keep = self._mlp_struct(weights, s_in, s_y, s_out)
        self._check(self.lib.sgpu_set_sgs_mlp(self._ctx, ctypes.byref(st)), "set_sgs_mlp")

    def set_sgs_fallback(self, bound=0.0, cs=0.0, ineg=1, enable=True):
        """Per-plane switch of the learned model to the eddy-viscosity model
        (dynamic when cs = 0) on planes where sum tau_ij S_ij > bound * sum
        |tau_ij S_ij| (predicted backscatter)."""
        self._check(self.lib.sgpu_set_sgs_fallback(self._ctx, int(bool(enable)), float(bound), float(cs), int(ineg)),
                    "set_sgs_fallback")

    def sgs_fallback_planes(self):
        """(planes (ny,) int: 1 where the last substep used the eddy-viscosity
        stress, sums (ny, 2): sum tau_ij S_ij and sum |tau_ij S_ij| per plane)."""
        planes = np.zeros(self.ny, np.int32)
        sums = np.zeros((self.ny, 2))
        self._check(self.lib.sgpu_sgs_fallback_planes(self._ctx, planes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                      _dp(sums)), "sgs_fallback_planes")
        return planes, sums

    def sgs_mlp_eval(self, weights, x, s_in=1.0, s_y=1.0, s_out=1.0):
        """The tensor-core MLP on feature rows x (n, 10) -> (n, 6)."""
        st, keep = self._mlp_struct(weights, s_in, s_y, s_out)
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], 6), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self._check(self.lib.sgpu_sgs_mlp_eval(self._ctx, ctypes.byref(st), x.ctypes.data_as(fp),
                                               y.ctypes.data_as(fp), x.shape[0]), "sgs_mlp_eval")
        return y

    def sgs_stress(self):
        """tau_ij of the last substep (iles = 2), shape (6, nz, ny, nx//2): 11 12 13 22 23 33."""
        shape = (6,) + self.shape
        re_ = np.empty(shape)
        im_ = np.empty(shape)
        self._check(self.lib.sgpu_download_sgs_stress(self._ctx, _dp(re_), _dp(im_)), "download_sgs_stress")
        return re_ + 1j * im_

    AMP_ROW = ("t", "urms", "vrms", "wrms", "omxrms", "omyrms", "omzrms", "omy2_k2", "uv", "e0", "hplus", "px",
               "re_bulk", "tau1", "tau2", "delta99", "delta_star", "theta", "w_bulk")

    def amplitudes(self):
        """Plane statistics and the amp.stat row of the current state
        (bla/boxamp.f, bla/wampbl.f): (amp array (20, ny) with amp[k-1, y-1] =
        amp(y, k), row as a dict keyed by AMP_ROW)."""
        amp = np.zeros((20, self.ny))
        row = np.zeros(19)
        self._check(self.lib.sgpu_amplitudes(self._ctx, _dp(amp), _dp(row)), "amplitudes")
        return amp, dict(zip(self.AMP_ROW, row))

    NXYS = 96

    def xys_sample(self, dtn=None):
        """Add one xy-statistics sample of the current state with weight dtn
        (default the time step) to the running sums (bla/boxxys.f as
        bla/bla.f:2069-2107 takes it)."""
        self._check(self.lib.sgpu_xys_sample(self._ctx, float(self.dt if dtn is None else dtn)), "xys_sample")

    def xys(self):
        """The running xy statistics: (xys, sumw) with xys[s-1, y, x] =
        xys(x+1, y+1, s) of the reference, shape (96, ny, nx)."""
        out = np.empty((self.NXYS, self.ny, self.nx))
        sw = np.zeros(1)
        self._check(self.lib.sgpu_xys_get(self._ctx, _dp(out), _dp(sw)), "xys_get")
        return out, float(sw[0])

    def xys_reset(self):
        self._check(self.lib.sgpu_xys_reset(self._ctx), "xys_reset")

    def sgs_mlp_train(self, params, adam_m, adam_v, adam_step, x, t, iters, lr):
        """Full-batch Adam training of the learned SGS model on the device
        (sgpu_sgs_mlp_train).  params, adam_m, adam_v: packed float32 (5254);
        x [n][10], t [n][6].  Returns (params, adam_m, adam_v, adam_step,
        loss, grad) after iters steps (loss and grad at the final weights)."""
        fp = ctypes.POINTER(ctypes.c_float)
        p = np.ascontiguousarray(params, np.float32).copy()
        m = np.ascontiguousarray(adam_m, np.float32).copy()
        v = np.ascontiguousarray(adam_v, np.float32).copy()
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        step = ctypes.c_int(int(adam_step))
        loss = ctypes.c_float()
        grad = np.empty(p.size, np.float32)
        self._check(self.lib.sgpu_sgs_mlp_train(self._ctx, p.ctypes.data_as(fp), m.ctypes.data_as(fp),
                                                v.ctypes.data_as(fp), ctypes.byref(step), x.ctypes.data_as(fp),
                                                t.ctypes.data_as(fp), x.shape[0], int(iters), float(lr),
                                                ctypes.byref(loss), grad.ctypes.data_as(fp)), "sgs_mlp_train")
        return p, m, v, step.value, loss.value, grad

    def pressure(self):
        """Pressure of the current state (bla/nonlinp.f + bla/linearp.f),
        complex (nz, ny, nx/2): Fourier x/z, physical y."""
        re_ = np.empty(self.shape)
        im_ = np.empty(self.shape)
        self._check(self.lib.sgpu_pressure(self._ctx, _dp(re_), _dp(im_)), "pressure")
        return re_ + 1j * im_

    def box_filter_sample(self, factor=4):
        """Training sample of the learned SGS model from the current state:
        (features (ny, nz/f, nx/f, 10), targets (ny, nz/f, nx/f, 6)), float32;
        see sgpu_box_filter_sample."""
        shape = (self.ny, self.nz // factor, self.nx // factor)
        feats = np.empty(shape + (10,), np.float32)
        tau = np.empty(shape + (6,), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self._check(self.lib.sgpu_box_filter_sample(self._ctx, int(factor), feats.ctypes.data_as(fp),
                                                    tau.ctypes.data_as(fp)), "box_filter_sample")
        return feats, tau

    KERNELS = ("zinv", "xpass", "zfwd", "cheb_fwd", "pencil", "mean", "cheb_inv", "other")

    def profile(self, enable=True):
        self._check(self.lib.sgpu_profile(self._ctx, int(enable)), "profile")

    def profile_read(self):
        n = len(self.KERNELS)
        ms = np.zeros(n)
        cnt = (ctypes.c_int * n)()
        self._check(self.lib.sgpu_profile_read(self._ctx, _dp(ms), cnt, n), "profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.KERNELS)}

    def launches(self):
        return int(self.lib.sgpu_launch_count(self._ctx))


class PinnedArray:
    """A numpy view of page-locked host memory allocated by the library."""

    def __init__(self, shape, dtype=np.float64):
        lib = load_library()
        self.lib = lib
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = ctypes.c_void_p()
        rc = lib.sgpu_host_alloc(n, ctypes.byref(self.ptr))
        if rc != 0:
            raise SimsonError("sgpu_host_alloc failed")
        buf = (ctypes.c_char * n).from_address(self.ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            self.lib.sgpu_host_free(self.ptr)
            self.ptr = None
