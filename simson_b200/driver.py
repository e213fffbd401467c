"""Host driver of a bla run on the GPU: the part of program bla
(bla/bla.f) around the two plane loops that this library replaces, for the
temporal channel.  Reads bla.i (and sgs.i), the initial field, steps, and
writes what the reference writes for such a run:

* start (bla/bla.f:960-1082, 1405-1478, 1562-1662): the field of namnin
  (bla/rdiscbl.f through simson_b200.ufile; re, xl, zl and t come from the
  file, as they do for a temporal run), the pressure gradient of the flow
  type (bla/bla.f:1622-1661: fltype 1 drives with the constant flux 4/3 or
  px = -(Re_tau/Re)^2, every other flow type has px = 0), for a spatial run
  (spat) the base flow (bla/bflow.f: bla/cbflow.f's Poiseuille or Couette
  profile, or the field of nambfl read as bla/rbflow.f does), the fringe
  (bla/ffun.f, bla/fring.f) and its time-step bound (bla/bla.f:1418-1431),
  the first time step (dt > 0 as given; dt <= 0: cflmax over the field's CFL
  rate, bla/getdt.f; either bounded by dtmax, bla/bla.f:1467), the LES model
  of sgs.i, prhs;
* every full step (nst substeps): with a variable time step, the next step's
  dt after the step's CFL evaluation, by the rule of bla/bla.f:2355-2380
  (cfl/cflmax above 10/9: dt cflmax/cfl, else dt (0.8 + 0.2 cflmax/cfl);
  at most dtmax; stretched to land on the next save time); the CFL stop
  (bla/wcflbl.f:93) through sgpu_get_scalars;
* the amp.stat line of bla/wampbl.f:276-278 when mod(it - 1 - nst, iamp) = 0
  (the state at the start of the step, as nonlinbl samples it), the velocity
  fields of the save times (bla/bla.f:2612-2660; bla/wdiscbl.f), then namnut
  at the end;
* stop (bla/bla.f:2800-2835): maxit substeps, t + dt/2 beyond tmax, wall-
  and CPU-time limits.

Options the library does not run stop with DeckError naming them
(simson_b200.blai.unsupported).  The xy statistics of ixys are sampled on the
device by sgpu_xys_sample; their file (xy.stat, bla/wxys.f) is not written
by this driver, so a deck that would take a sample stops with DeckError.

Usage: python -m simson_b200.driver DECK_DIR [--grid NXxNYxNZ]
       [--precision fp64|mixed] [--max-steps N]
"""
from __future__ import annotations

import argparse
import math
import os
import time

from . import blai, ufile
from .bla import FP64, MIXED, Channel, base_flow, base_flow_from_fields


def fortran_e(v, w=25, d=16, e=3):
    """A value in Fortran's Ew.dEe edit descriptor (0.ddd...E+eee)."""
    if not math.isfinite(v):
        return str(v).rjust(w)
    if v == 0.0:
        return (f"{0.0:.{d}f}" + "E+" + "0" * e).rjust(w)
    x = math.floor(math.log10(abs(v))) + 1
    m = round(v / 10.0 ** x, d)
    if abs(m) >= 1.0:  # rounding up to the next decade
        m /= 10.0
        x += 1
    s = f"{m:.{d}f}"
    return (s + ("E+" if x >= 0 else "E-") + f"{abs(x):0{e}d}").rjust(w)


def amp_line(row):
    """One amp.stat line (bla/wampbl.f:276-278: 19(e25.16e3, tr1))."""
    return "".join(fortran_e(float(row[k])) + " " for k in Channel.AMP_ROW)


def next_dt(dtn, cfl, cflmax, dtmax, t, tsave_next, tmax):
    """dtnp1 of bla/bla.f:2355-2380."""
    if tmax > 0:
        tleft = min(tmax, tsave_next) - t - dtn
    else:
        tleft = tsave_next - t - dtn
    if cfl / cflmax > 10.0 / 9.0:
        dtnp1 = dtn * cflmax / cfl
    else:
        dtnp1 = dtn * (0.8 + 0.2 * cflmax / cfl)
    dtnp1 = min(dtnp1, dtmax)
    if 0.5 * dtnp1 < tleft < 4.0 * dtnp1:
        dtnp1 = tleft / math.trunc(tleft / dtnp1 + 1.0)
    return dtnp1


def run(deck_dir, grid=None, precision="fp64", device=0, max_steps=None, log=print):
    """Run the deck in deck_dir.  grid (nx, ny, nz) overrides the file's size
    (varsiz).  Returns a summary dict (steps, t, dt, it, px, files written)."""
    b = blai.read_bla_i(os.path.join(deck_dir, "bla.i"))
    bad = blai.unsupported(b)
    if bad:
        raise blai.DeckError("options this library does not run: " + ", ".join(bad))
    les = blai.read_sgs_i(os.path.join(deck_dir, "sgs.i")) if b.sgs else None
    if b.iamp > 0 and b.iamp % b.nst:
        # nonlinbl samples at any substep with mod(it-1-nst, iamp) = 0; this
        # driver samples at step boundaries only
        raise blai.DeckError(f"iamp = {b.iamp} is not a multiple of nst = {b.nst}")
    init = blai.deck_path(deck_dir, b.namnin)
    head = ufile.read_header(init)
    fltype = head["fltype"]
    if fltype not in (1, 2, 4, 5) or (b.spat and fltype not in (4, 5)):
        raise blai.DeckError(f"flow type {fltype}" + (" in a spatial run" if b.spat else "") +
                             ": this library steps the channel (fltype 1, 2; spatial 4, 5)")
    nx, ny, nz = grid or (head["nx"], head["nyp"], head["nzc"])
    _, fields = ufile.read_u(init, m=3, nx=nx, nyp=ny, nz=nz, varsiz=b.varsiz)
    re, xl, zl, t0 = head["re"], head["xl"], head["zl"], head["t"]
    nst = b.nst
    # pressure gradient (bla/bla.f:1622-1661)
    cflux = b.cflux and fltype == 1
    px = (-2.0 / re) if cflux else (-(b.retau / re) ** 2 if fltype == 1 else 0.0)
    dtmax = b.dtmax
    if b.spat:  # the fringe's bound on the time step (bla/bla.f:1418-1431)
        dtmax = min(dtmax, (1.75 if nst == 3 else 1.96) / b.fmax)
    dt0 = min(b.dt, dtmax) if b.dt > 0 else 1.0
    ch = Channel(nx, ny, nz, re, xl, zl, dt0, cflux=cflux, px=px, icfl=b.icfl, nst=nst,
                 rot=b.rot, precision=MIXED if precision == "mixed" else FP64, device=device)
    written = []
    wall0, cpu0 = time.time(), time.process_time()
    try:
        if les is not None and les.iles:
            ch.set_les(iles=les.iles, cutoff_inv=les.cutoff_inv, iord=les.iord, chi=les.chi, cs=les.cs,
                       ineg=les.ineg)
        if b.spat:
            nxp = 3 * nx // 2
            if b.rbfl:
                _, bf = ufile.read_u(blai.deck_path(deck_dir, b.nambfl), m=3, nx=nx, nyp=ny, nz=nz, varsiz=True)
                ch.set_base_flow(*base_flow_from_fields(*bf, nxp=nxp))
            else:
                ch.set_base_flow(*base_flow(fltype, ny, nxp))
            ch.set_fringe(b.fstart, b.fend, b.frise, b.ffall, b.fmax)
        ch.set_velocity(*fields)
        dtn = dt0
        if b.vart:
            dtn = min(b.cflmax / ch.cfl_rate(), dtmax)  # getdt, then bla/bla.f:1467
            ch.set_dt(dtn)
            log(f"First time step      : {dtn}")
        ch.prhs()
        tsave = list(b.tsave) + [1.0e30]
        names = list(b.nmsave)
        isave = 0  # the first save time not yet passed (bla/bla.f:1678-1686)
        while isave < len(names) and t0 >= tsave[isave]:
            isave += 1
        amp_f = open(blai.deck_path(deck_dir, b.namamp), "w") if b.iamp > 0 else None
        it, steps = 1, 0
        sc = ch.scalars()
        t = t0
        try:
            while True:
                t = t0 + ch.scalars()["t"]
                if amp_f is not None and (it - 1 - nst) % b.iamp == 0:
                    _, row = ch.amplitudes()
                    amp_f.write(amp_line(dict(row, t=t)) + "\n")
                if b.ixys > 0 and (it - 1 - nst) % b.ixys == 0 and t >= b.txys:
                    raise blai.DeckError("xy statistics would be sampled: the xy.stat writer is not built")
                if b.vart:
                    ch.substeps(nst - 1)
                    sc = ch.scalars()  # the CFL of this step's first substep; stops as wcflbl.f:93
                    dtnp1 = next_dt(dtn, sc["cfl"], b.cflmax, dtmax, t, tsave[isave], b.tmax)
                    ch.set_dt(dtnp1)
                    ch.substeps(1)
                    dtn = dtnp1
                else:
                    ch.step(1)
                it += nst
                steps += 1
                sc = ch.scalars()
                t = t0 + sc["t"]
                if isave < len(names) and t + 0.5 * dtn > tsave[isave]:
                    path = blai.deck_path(deck_dir, names[isave])
                    ufile.write_u(path, ch.state(3), re, xl, zl, t)
                    written.append(path)
                    log(f"Saved {names[isave]} at t = {t}")
                    isave += 1
                stop = None
                if b.wallmax > 0 and time.time() - wall0 > b.wallmax:
                    stop = "wall time"
                if b.cpumax > 0 and time.process_time() - cpu0 > b.cpumax:
                    stop = "cpu time"
                if b.maxit > 0 and it - 1 >= b.maxit:
                    stop = "iterations"
                if b.tmax > 0 and t + 0.5 * dtn > b.tmax:
                    stop = "integration time"
                if max_steps is not None and steps >= max_steps:
                    stop = "the driver's step limit"
                if stop:
                    log(f"STOP DUE TO {stop.upper()} (t = {t}, {steps} steps)")
                    break
        finally:
            if amp_f is not None:
                amp_f.close()
        out = blai.deck_path(deck_dir, b.namnut)
        ufile.write_u(out, ch.state(3), re, xl, zl, t)
        written.append(out)
        return dict(steps=steps, t=t, dt=dtn, it=it, written=written, px=sc["px"])
    finally:
        ch.close()


def main():
    ap = argparse.ArgumentParser(description="run a bla deck (bla.i, sgs.i, the initial .u) on the GPU")
    ap.add_argument("deck")
    ap.add_argument("--grid", default=None, help="NXxNYxNZ (default: the initial field's)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--max-steps", type=int, default=None)
    a = ap.parse_args()
    grid = tuple(int(v) for v in a.grid.split("x")) if a.grid else None
    print(run(a.deck, grid, a.precision, max_steps=a.max_steps))


if __name__ == "__main__":
    main()
