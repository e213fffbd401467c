"""Readers of the reference's input decks: ``bla.i`` (version 20070716) and
``sgs.i`` (version 20060909), record by record in the order
bla/rparambl.f:150-1880 and bla/rparamles.f:31-90 read them.

Reading rules of the reference:

* before every record, ``comment`` (bla/comment.f) skips the lines whose first
  non-blank character is ``#``; blank lines are skipped by the list-directed
  read itself;
* a list-directed record (``read(10,*) x``) takes the first value of its line
  (blank or comma separated; logicals as ``.true.``, ``t``, ``.f.`` ...;
  reals with ``d`` or ``e`` exponents); a character record
  (``read(10,'(a)') name``) takes the whole line;
* the records that follow depend on earlier values (``cflux``, ``pert``,
  ``suction``, ``spat``, ``isfd``, ``imhd``, ``loctyp``, ``tripf``, ``wbci``,
  ``iamp``, ``iext``, ``ixys``, ``msave``, ``mwave``, ``npl``), as in
  rparambl.f; after the last record the derived values are set as
  rparambl.f:1862-1864, 1995-2017 do (``icfl`` in whole steps, ``vart``,
  ``dtmax``, ``cflmax``).

Options whose physics this library does not implement (perturbation mode,
forcing in the fringe other than the damping to the base flow, tabulated
free-stream velocities, suction, localized forcing, trips, wall roughness or
jets, MHD, SFD, scalars, two-point correlations, time series) are reported by
:func:`unsupported` or, where the records that follow them are not read
here, stop the reading with DeckError naming the option.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

BLA_VERSION = 20070716
SGS_VERSION = 20060909


class DeckError(ValueError):
    """An input deck the reference would reject, or one that asks for an
    option this library does not run (named in the message)."""


class _Deck:
    """Line reader with comment(10) and the two record forms."""

    def __init__(self, path):
        self.path = path
        with open(path) as f:
            self.lines = f.read().splitlines()
        self.i = 0

    def _comment(self):
        while self.i < len(self.lines):
            s = self.lines[self.i].strip()
            if s and not s.startswith("#"):
                return
            self.i += 1
        raise DeckError(f"{self.path}: end of file before a required record")

    def text(self):
        """read(10,'(a)'): the whole line, blanks around it dropped."""
        self._comment()
        s = self.lines[self.i].strip()
        self.i += 1
        return s

    def _token(self):
        self._comment()
        line = self.lines[self.i]
        self.i += 1
        tok = line.replace(",", " ").split()
        if not tok or tok[0].startswith("/"):
            raise DeckError(f"{self.path}:{self.i}: no value on the line")
        return tok[0], self.i

    def int(self):
        t, ln = self._token()
        try:
            return int(t)
        except ValueError:
            try:
                v = float(t.lower().replace("d", "e"))
            except ValueError:
                raise DeckError(f"{self.path}:{ln}: expected an integer, got {t!r}") from None
            if v != int(v):
                raise DeckError(f"{self.path}:{ln}: expected an integer, got {t!r}")
            return int(v)

    def real(self):
        t, ln = self._token()
        try:
            return float(t.lower().replace("d", "e"))
        except ValueError:
            raise DeckError(f"{self.path}:{ln}: expected a real, got {t!r}") from None

    def logical(self):
        t, ln = self._token()
        s = t.lower().lstrip(".")
        if s[:1] == "t":
            return True
        if s[:1] == "f":
            return False
        raise DeckError(f"{self.path}:{ln}: expected a logical, got {t!r}")


@dataclass
class BlaInput:
    version: int = BLA_VERSION
    namnin: str = ""
    namnut: str = ""
    tmax: float = 0.0
    maxit: int = 0
    cpumax: float = 0.0
    wallmax: float = 0.0
    write_inter: bool = False
    dt: float = 0.0
    nst: int = 3
    cflmaxin: float = 0.8
    xl: float = 0.0
    varsiz: bool = False
    rot: float = 0.0
    cflux: bool = True
    retau: float = 0.0
    pert: bool = False
    lin: bool = False
    bf3: bool = False
    ibc: int = 0
    cim: bool = False
    icorr: int = 0
    gall: bool = False
    suction: bool = False
    spat: bool = False
    tabfre: bool = False
    rbfl: bool = False
    nambfl: str = ""
    fmax: float = 0.0
    fstart: float = 0.0
    fend: float = 0.0
    frise: float = 0.0
    ffall: float = 0.0
    ampob: float = 0.0
    amp2d: float = 0.0
    cdev: float = 0.0
    sgs: bool = False
    isfd: int = 0
    imhd: int = 0
    loctyp: int = 0
    tripf: bool = False
    wbci: int = 0
    icfl: int = 0
    iamp: int = 0
    namamp: str = ""
    fileurms: bool = False
    longli: bool = False
    iext: int = 0
    namext: str = ""
    ixys: int = 0
    namxys: str = ""
    ixyss: int = 0
    txys: float = 0.0
    corrf: bool = False
    corrf_x: bool = False
    serf: bool = False
    msave: int = 0
    tsave: list = field(default_factory=list)
    nmsave: list = field(default_factory=list)
    mwave: int = 0
    npl: int = 0
    # derived (rparambl.f:1862-1864, 1995-2017)
    vart: bool = False
    dtmax: float = 1.0e30
    cflmax: float = 0.0


@dataclass
class SgsInput:
    version: int = SGS_VERSION
    iles: int = 1
    cutoff_inv: float = 1.5
    iord: int = 5
    chi: float = 0.2
    cs: float = 0.0
    ineg: int = 1
    ihighorder: int = 2
    prt: float = 0.6


# records of the localized-forcing branches (rparambl.f:827-1153) and of the
# wall boundary conditions (rparambl.f:1202-1435) that are plain values
_LOCTYP_RECORDS = {2: 13, 6: 7, 7: 6, 8: 9, 10: 3, 12: 5, 13: 8}
_WBCI_RECORDS = {0: 0, 1: 8, 2: 14, 3: 10, 4: 8, 5: 11, -2: 5}


def read_bla_i(path, scalar=0, mxys=1) -> BlaInput:
    """Parse a bla.i.  scalar, mxys: the par.f constants of the build (the
    records per passive scalar and per xy-statistics box)."""
    d = _Deck(path)
    b = BlaInput()
    b.version = d.int()
    if b.version != BLA_VERSION:
        raise DeckError(f"Wrong version of bla.i, now: {b.version}, bla version is: {BLA_VERSION} (stop 345431)")
    b.namnin = d.text()
    b.namnut = d.text()
    b.tmax = max(d.real(), 0.0)
    b.maxit = max(d.int(), 0)
    b.cpumax = max(d.real(), 0.0)
    b.wallmax = max(d.real(), 0.0)
    b.write_inter = d.logical()
    b.dt = d.real()
    b.nst = d.int()
    b.cflmaxin = d.real()
    b.xl = d.real()
    b.varsiz = d.logical()
    b.rot = d.real()
    b.cflux = d.logical()
    if not b.cflux:
        b.retau = d.real()
    b.pert = d.logical()
    if b.pert:
        b.lin = d.logical()
        b.bf3 = d.logical()
        if b.bf3:
            d.text()
    b.ibc = d.int()
    if scalar:
        raise DeckError("passive scalars (the tbc records) are not built")
    b.cim = d.logical()
    if b.cim:
        b.icorr = d.int()
    b.gall = d.logical()
    b.suction = d.logical()
    if b.suction:
        if not d.logical():  # asbl
            d.real()  # vsuc
    b.spat = d.logical()
    if b.spat:
        # rparambl.f:547-686: base flow source, fringe, forcing in the fringe
        b.tabfre = d.logical()
        if b.tabfre:
            raise DeckError("tabulated free-stream velocity (tabfre) is not built")
        b.rbfl = d.logical()
        if b.rbfl:
            b.nambfl = d.text()
        b.fmax = d.real()
        b.fstart = d.real()
        b.fend = d.real()
        b.frise = d.real()
        b.ffall = d.real()
        b.ampob = d.real()
        b.amp2d = d.real()
        if d.logical():
            raise DeckError("Orr-Sommerfeld forcing in the fringe (osmod) is not built")
        if d.logical():
            raise DeckError("streak forcing in the fringe (streak) is not built")
        if d.logical():
            raise DeckError("waves in the fringe (waves) is not built")
        # rparambl.f:1898-1912
        if (b.fstart >= b.fend or b.frise <= 0.0 or b.ffall <= 0.0 or b.fmax <= 0.0
                or abs(b.fstart) > 0.5 * b.xl or abs(b.fend) > 0.5 * b.xl):
            raise DeckError("fmax, frise, ffall must be positive and fstart < fend in -xl/2 to xl/2")
    elif not b.suction:
        b.cdev = d.real()
    b.sgs = d.logical()
    b.isfd = d.int()
    if b.isfd >= 1:
        if not d.logical():  # sfdzero
            d.text()
        d.real()
        d.real()
    b.imhd = d.int()
    if b.imhd == 1:
        for _ in range(4):
            d.real()
    elif b.imhd != 0:
        raise DeckError(f"imhd = {b.imhd} is neither 0 nor 1")
    b.loctyp = d.int()
    if b.loctyp == 1:
        for _ in range(6):
            d.real()
        if d.real() < 0:  # fpds4 < 0: fp1 follows
            d.real()
        d.real()
    elif b.loctyp != 0:
        n = _LOCTYP_RECORDS.get(b.loctyp)
        if n is None:
            raise DeckError(f"localized forcing loctyp = {b.loctyp} is not read by this reader")
        for _ in range(n):
            d.real()
    b.tripf = d.logical()
    if b.tripf:
        for _ in range(8):
            d.real()
    b.wbci = d.int()
    if b.wbci == -1:
        d.text()  # wallroughinput
    else:
        n = _WBCI_RECORDS.get(b.wbci)
        if n is None:
            raise DeckError(f"wall boundary condition wbci = {b.wbci} is not read by this reader")
        for _ in range(n):
            d.real()
    b.icfl = d.int()
    b.iamp = d.int()
    if b.iamp > 0:
        b.namamp = d.text()
        b.fileurms = d.logical()
    b.longli = d.logical()
    b.iext = d.int()
    if b.iext > 0:
        b.namext = d.text()
    ixys = max(0, d.int())
    if ixys > 0:
        ixys = max(ixys, b.nst) // b.nst * b.nst
    b.ixys = ixys
    if ixys > 0:
        b.namxys = d.text()
        ixyss = max(0, d.int())
        b.txys = d.real()
        if ixyss > 0:
            ixyss = max(ixyss, b.nst) // b.nst * b.nst
        b.ixyss = ixyss
        if mxys > 1:
            d.real()  # xysp
        b.corrf = d.logical()
        if b.corrf:
            raise DeckError("two-point correlations (corrf) are not built")
        b.corrf_x = d.logical()
        if b.corrf_x:
            raise DeckError("two-point correlations (corrf_x) are not built")
        b.serf = d.logical()
        if b.serf:
            raise DeckError("time series (serf) are not built")
    msave = d.int()
    if msave == 100000:
        raise DeckError("periodic saving (msave = 100000) is not read by this reader")
    if msave < 0:
        raise DeckError("saving by frequency (msave < 0) is not read by this reader")
    for _ in range(msave):
        b.tsave.append(d.real())
        b.nmsave.append(d.text())
    b.msave = msave
    b.mwave = d.int()
    if b.mwave > 0:
        d.text()
        for _ in range(b.mwave):
            d.text()
    b.npl = d.int()
    if b.npl > 0:
        d.int()
        for _ in range(b.npl):
            d.real()
            d.real()
            d.int()
            d.text()
    # adjustments of rparambl.f:1862-1864 and 1995-2017
    if b.nst not in (3, 4):
        raise DeckError("Stop: nst must be 3 for 3-stage RK3 or 4 for 4-stage RK3.")
    if 0 < b.icfl < b.nst:
        b.icfl = b.nst
    if b.icfl > 0:
        b.icfl = min(b.icfl // b.nst * b.nst, 3 * b.nst)
    if b.dt <= 0 and b.icfl <= 0:
        b.icfl = b.nst
    b.vart = b.dt <= 0
    b.dtmax = -b.dt if b.dt < 0 else 1.0e30
    b.cflmax = b.cflmaxin * (math.sqrt(3.0) if b.nst == 3 else math.sqrt(8.0))
    return b


def read_sgs_i(path) -> SgsInput:
    """Parse an sgs.i (bla/rparamles.f:31-90): iles 0 none, 1 ADM-RT (cutoff
    1/fraction, order, chi), 2 eddy viscosity (cs; ineg when cs = 0), 3 HPF
    eddy viscosity (cutoff, order, cs; ineg when cs = 0)."""
    d = _Deck(path)
    s = SgsInput()
    s.version = d.int()
    if s.version != SGS_VERSION:
        raise DeckError(f"Wrong version of sgs.i, now: {s.version}, bla version is: {SGS_VERSION} (stop 345432)")
    s.iles = d.int()
    if s.iles == 1:
        s.cutoff_inv = d.real()
        s.iord = d.int()
        s.chi = d.real()
    elif s.iles == 2:
        s.cs = d.real()
        if s.cs == 0:
            s.ineg = d.int()
    elif s.iles == 3:
        s.cutoff_inv = d.real()
        s.iord = d.int()
        s.cs = d.real()
        if s.cs == 0:
            s.ineg = d.int()
    elif s.iles != 0:
        raise DeckError(f"sgs.i: unknown iles = {s.iles}")
    return s


def unsupported(b: BlaInput):
    """The options of a parsed deck that this library's channel step does not
    run (empty: the deck runs)."""
    checks = [(b.pert, "perturbation equations (pert)"), (b.ibc != 0, f"boundary condition ibc = {b.ibc}"),
              (b.cim, "Chebyshev integration method (cim)"), (b.gall, "Galilean transformation (gall)"),
              (b.suction, "wall suction"), (b.cdev != 0.0, "temporal development velocity (cdev)"),
              (b.isfd != 0, "selective frequency damping (isfd)"), (b.imhd != 0, "MHD (imhd)"),
              (b.loctyp != 0, f"localized forcing loctyp = {b.loctyp}"), (b.tripf, "trip forcing"),
              (b.wbci != 0, f"wall boundary condition wbci = {b.wbci}"),
              (b.ampob != 0.0 or b.amp2d != 0.0, "wave forcing in the fringe (ampob, amp2d)"),
              (b.gall and b.spat, "Galilean transformation of a spatial run"),
              (b.longli, "y-dependent amplitude file (longli)"),
              (b.iext > 0, "extremum file (iext)"), (b.mwave > 0, "wavenumber output (mwave)"),
              (b.npl > 0, "plane output (npl)")]
    return [what for bad, what in checks if bad]


def deck_path(deck_dir, name):
    return name if os.path.isabs(name) else os.path.join(deck_dir, name)
