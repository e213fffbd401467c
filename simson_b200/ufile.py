"""The reference's velocity field file (``.u``): written by bla/wdiscbl.f,
read by bla/rdiscbl.f (and its pressure file ``.p`` of bla/wdiscp.f); the checkpoint of a run (a restart at a full step is
exact in exact arithmetic: the first RK stage has b_1 = 0, so the partial
right-hand sides are rebuilt from u by prhs).

Format (gfortran unformatted sequential, little-endian, 4-byte record
markers before and after every record; real = 8 bytes, integer and logical
= 4 bytes), for scalar = 0:

  re, pou(.false.), xl, zl, t, xs(0.)            (wdiscbl.f:50-56)
  nx, nyp, nzc, nfzsym                           (:57)
  fltype, dstar                                  (:58)
  [rlam | rlam, spanv | bstart, blength | ...]   (:59-64, by fltype)
  then for each of the m fields, each stored kz plane z = 1..nzc, each y =
  1..nyp: one record of nx reals, re/im interleaved for kx = 0..nx/2-1
  (:112-136).

Fields at this interface are complex arrays of shape (nz, nyp, nx/2) in the
storage order of kz (0..nz/2, -nz/2+1..-1), as simson_b200.bla.Channel
uploads them.
"""
from __future__ import annotations

import struct

import numpy as np

# extra header record of each flow type (wdiscbl.f:59-64; scalar = 0)
_EXTRA = {-1: ("rlam",), -2: ("rlam", "spanv"), 4: ("bstart", "blength"), 5: ("bstart", "blength"),
          6: ("bstart", "blength", "rlam", "spanv"), 7: ("bstart", "blength", "rlam", "spanv"),
          8: ("bstart", "blength", "rlam", "spanv"), 9: ("bstart", "blength", "rlam", "spanv"),
          20: (), -20: ()}
# flow types rdiscbl accepts (rdiscbl.f:180-188)
_VALID = set(range(-3, 0)) | set(range(1, 10)) | {20, -20}


# extra header record of the pressure file (bla/wdiscp.f, the .p file): every
# fltype >= 6 writes bstart, blength, rlam, spanv, 20 included
def _extra_names(fltype, pressure_file=False):
    if not pressure_file:
        return _EXTRA.get(fltype)
    if fltype >= 6:
        return ("bstart", "blength", "rlam", "spanv")
    return {-1: ("rlam",), -2: ("rlam", "spanv"), 4: ("bstart", "blength"), 5: ("bstart", "blength")}.get(fltype)


class UFileError(ValueError):
    """A .u file the reader cannot take (the cases where rdiscbl stops)."""


def _record(f, payload: bytes):
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def write_p(path, p, re, xl, zl, t, dstar=1.0, fltype=1, **extra):
    """Write a pressure field (complex (nz, nyp, nx/2), e.g. from
    Channel.pressure) as bla/wdiscp.f does: the header of the velocity file
    and the one field (slot 8).  The reference names the file after the
    velocity file with '.p' appended; path is the full name."""
    write_u(path, [p], re, xl, zl, t, dstar, fltype, _pressure_file=True, **extra)


def write_u(path, fields, re, xl, zl, t, dstar=1.0, fltype=1, _pressure_file=False, **extra):
    """Write fields (m complex arrays (nz, nyp, nx/2)) as wdiscbl does with
    xs = zs = 0 (no box shift) and gall = .false.."""
    fields = [np.asarray(q) for q in fields]
    nz, nyp, nx2 = fields[0].shape
    nx = 2 * nx2
    if fltype not in _VALID:
        raise UFileError(f"flow type {fltype} not writable")
    with open(path, "wb") as f:
        _record(f, struct.pack("<di4d", re, 0, xl, zl, t, 0.0))
        _record(f, struct.pack("<4i", nx, nyp, nz, 0))
        _record(f, struct.pack("<id", fltype, dstar))
        names = _extra_names(fltype, _pressure_file)
        if names is not None:
            _record(f, struct.pack("<%dd" % len(names), *[float(extra.get(k, 0.0)) for k in names]))
        row = np.empty(nx, "<f8")
        for q in fields:
            if q.shape != (nz, nyp, nx2):
                raise UFileError("fields of different shapes")
            for z in range(nz):
                for y in range(nyp):
                    row[0::2] = q[z, y].real
                    row[1::2] = q[z, y].imag
                    _record(f, row.tobytes())


class _Reader:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.buf = f.read()
        self.pos = 0

    def record(self) -> bytes:
        b = self.buf
        if self.pos + 4 > len(b):
            raise UFileError("truncated file: record marker missing")
        (n,) = struct.unpack_from("<i", b, self.pos)
        if n < 0 or self.pos + 8 + n > len(b):
            raise UFileError("truncated file or corrupt record marker")
        payload = b[self.pos + 4:self.pos + 4 + n]
        (n2,) = struct.unpack_from("<i", b, self.pos + 4 + n)
        if n2 != n:
            raise UFileError("corrupt record: leading and trailing markers differ")
        self.pos += 8 + n
        return payload


def _cheb_regrid(q, nyp_out):
    """rdiscbl.f:343-372: a field on nypin Gauss-Lobatto points (axis 1)
    expanded in Chebyshev polynomials and evaluated on nyp_out points."""
    nin = q.shape[1]
    j = np.arange(nin)
    theta = np.pi * j / (nin - 1)
    # coefficients a_k = 2/(N) sum'' q_j cos(k theta_j), N = nin - 1
    w = np.ones(nin)
    w[0] = w[-1] = 0.5
    cosm = np.cos(np.outer(j, theta))                  # [k, j]
    a = (2.0 / (nin - 1)) * np.einsum("kj,zjx->zkx", cosm * w[None, :], q)
    a[:, 0] *= 0.5
    a[:, -1] *= 0.5
    theta_out = np.pi * np.arange(nyp_out) / (nyp_out - 1)
    return np.einsum("yk,zkx->zyx", np.cos(np.outer(theta_out, j)), a)


def read_header(path, pressure_file=False):
    """The header records of a .u (or .p) file as read_u returns them,
    without the fields."""
    head, _ = read_u(path, m=0, pressure_file=pressure_file)
    return head


def read_u(path, m=3, nx=None, nyp=None, nz=None, varsiz=True, pressure_file=False):
    """Read a .u file.  Returns (header dict, list of m fields (nz, nyp,
    nx/2)).  With a target size different from the file's, as rdiscbl does
    with varsiz: x and z modes truncated or zero-padded, y refined (never
    reduced) by Chebyshev re-expansion; the kz = -nzin/2 mode of an even
    file grid, which is not an oddball on a larger grid, is zeroed.  Raises
    UFileError where rdiscbl stops.  pressure_file: a .p file of wdiscp
    (its header record by flow type; read it with m = 1)."""
    r = _Reader(path)
    rec = r.record()
    if len(rec) != 44:
        raise UFileError("first header record has the wrong length (scalar fields are not supported)")
    re, pou, xl, zl, t, xs = struct.unpack("<di4d", rec)
    rec = r.record()
    if len(rec) != 16:
        raise UFileError("grid record has the wrong length")
    nxin, nypin, nzcin, nfzsin = struct.unpack("<4i", rec)
    if nxin < 2 or nxin % 2 or nypin < 2 or nzcin < 1:
        raise UFileError(f"impossible grid ({nxin}, {nypin}, {nzcin})")
    rec = r.record()
    if len(rec) < 12:
        raise UFileError("flow-type record has the wrong length")
    fltype, dstar = struct.unpack("<id", rec[:12])
    if fltype not in _VALID:
        raise UFileError(f"the file does not contain a known flow type: {fltype}")
    head = dict(re=re, pou=bool(pou), xl=xl, zl=zl, t=t, xs=xs, nx=nxin, nyp=nypin, nzc=nzcin, nfzsym=nfzsin,
                fltype=fltype, dstar=dstar)
    names = _extra_names(fltype, pressure_file)
    if names is not None:
        rec = r.record()
        if len(rec) != 8 * len(names):
            raise UFileError(f"flow-type {fltype} header record of the wrong length")
        vals = struct.unpack("<%dd" % len(names), rec)
        head.update(zip(names, vals))
    if nfzsin != 0:
        raise UFileError("z-symmetric fields (nfzsym = 1) are not supported")
    nx = nxin if nx is None else nx
    nyp = nypin if nyp is None else nyp
    nz = nzcin if nz is None else nz
    if (nx, nyp, nz) != (nxin, nypin, nzcin) and not varsiz:
        raise UFileError("the file has a size other than the program")
    if nypin > nyp:
        raise UFileError("resolution cannot be reduced in y")
    nxr = min(nx, nxin)
    fields = []
    walls = []
    for _ in range(m):
        q = np.zeros((nz, nypin, nx // 2), complex)
        for z in range(nz):
            if nz > 1 and (nzcin + 1) // 2 <= z < nz - nzcin // 2:
                pass  # modes the file does not have (rdiscbl.f:289-298)
            else:
                for y in range(nypin):
                    rec = r.record()
                    if len(rec) != 8 * nxin:
                        raise UFileError("data record of the wrong length")
                    row = np.frombuffer(rec, "<f8", nxr)
                    q[z, y, :nxr // 2] = row[0::2] + 1j * row[1::2]
            if z == nz // 2 - 1 or nz == 1:
                for _zs in range(nz, nzcin):  # modes the program does not keep
                    for _y in range(nypin):
                        r.record()
        walls.append((q[0, 0, 0].real, q[0, -1, 0].real))  # the mean mode at y = +1 and -1
        if nypin < nyp:
            q = _cheb_regrid(q, nyp)
        if nz > nzcin and nzcin % 2 == 0:
            q[nz - nzcin // 2] = 0.0  # the file's -nzin/2 mode (rdiscbl.f:373-385)
        fields.append(q)
    # wall velocities of the mean mode, as read (rdiscbl.f:306-309)
    if not walls:
        return head, fields
    head["u0upp"], head["u0low"] = walls[0]
    if m >= 3:
        head["w0upp"], head["w0low"] = walls[2]
    return head, fields
