"""Recipe that builds the reference oracle ``oracle/_ref/<grid>/libsimson_ref.so``.

TEST INFRASTRUCTURE ONLY (see ``oracle/f77c.py``).  The product never loads it.

It reads the reference's Fortran sources where they lie (``$SIMSON_REFERENCE``,
default the read-only reference checkout), edits only the compile-time grid
in ``par.f`` exactly as the reference's own instructions say to do per case
(nx, ny, nz, nthread, and pressure = 0, or 1 for the pressure variant in
``oracle/_ref/<grid>_p``), translates the hot-path units to C with
``oracle/f77c.py`` and compiles them, together with ``oracle/ref_harness.c``,
with ``gcc -O3 -fopenmp``.  Nothing derived from the reference is written
outside ``oracle/_ref/`` (git-ignored).

Translated units (reference file: what it contributes):
  bla/bla.f         declarations of the driver state + these statement ranges:
                    849 rkcoeff call, 1080-1082 preprbl call, 1407-1416 getdt (variable
                    time step), 1466-1478 first-step
                    RK factors, 1562-1569 prhs call, 1622-1662 channel px/mflux init,
                    1796-1797 substep time, 1819-1826 box shift, 2251-2288 the
                    nonlinbl plane loop (OpenMP), 2349-2351 wcflbl, 2355-2380 the next
                    step's time step of a variable-step run, 2384-2397 RK
                    weights, 2433-2475 the linearbl plane loop (OpenMP), 2598 it=it+1
  bla/nonlinbl.f advection.f boxcfl.f fft2db.f fft2df.f getxz.f putxz.f   (step 2)
  bla/linearbl.f getxy.f putxy.f setmacrhs.f trid.f dcheb.f evald.f evalbc.f
                 solvbc.f                                                  (step 3)
  bla/prhs.f preprbl.f rkcoeff.f wcflbl.f getdt.f cvecfft_acc.f            (startup, CFL, FFTs)
  bla/boxamp.f                                                             (plane statistics)
  bla/boxxys.f xzsh.f + bla.f 2069-2107                                    (xy statistics)
  bla/nonlinp.f linearp.f crhsc.f setmac.f tridc.f icheb.f + bla.f 2486-2527 (pressure)
  bla/init_filter.f lpf_y.f hpf_y.f bandsolver.f + bla.f 1489-1545         (ADM-RT LES filters)
  bla/les.f sgs_stress.f filter_cutoff.f + bla.f 1945-2020                 (eddy-viscosity LES)
  bla/fring.f fringp.f ffun.f step.f bflow.f cbflow.f + bla.f 1338-1374 (base flow),
                 2166-2175 (fringe function)                               (spatial channel)
For grids up to SMAG_MAX_POINTS the driver's compile-time switch iiles_smag
(bla/bla.f:28) is set to 1, as the reference instructs for dynamic
Smagorinsky runs, so that its SGS-stress arrays exist.
Everything else those units call (dynamic SGS models, forcing, MPI, timers, ...) is
emitted as a stub that aborts if reached; the timers ``ctim``/``wall_time``
are no-ops.  The channel configuration never reaches a stub.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from f77c import translate  # noqa: E402

REF_ROOT = os.environ.get("SIMSON_REFERENCE", "/root/reference")
REF_BLA = os.path.join(REF_ROOT, "bla")
OUT_ROOT = os.path.join(HERE, "_ref")

UNIT_FILES = [
    "nonlinbl.f", "advection.f", "boxcfl.f", "fft2db.f", "fft2df.f", "getxz.f", "putxz.f",
    "linearbl.f", "getxy.f", "putxy.f", "setmacrhs.f", "trid.f", "dcheb.f", "evald.f",
    "evalbc.f", "solvbc.f", "prhs.f", "preprbl.f", "rkcoeff.f", "wcflbl.f", "cvecfft_acc.f", "boxamp.f",
    "init_filter.f", "lpf_y.f", "hpf_y.f", "bandsolver.f",
    "les.f", "sgs_stress.f", "filter_cutoff.f", "boxxys.f", "xzsh.f",
    "nonlinp.f", "linearp.f", "crhsc.f", "setmac.f", "tridc.f", "icheb.f", "getdt.f",
    "fring.f", "fringp.f", "ffun.f", "step.f", "bflow.f", "cbflow.f",
]

MAIN_RANGES = [
    ("bla_rkcoeff", 849, 849),
    ("bla_preprbl", 1080, 1082),
    ("bla_getdt", 1407, 1416),
    ("bla_firststep", 1466, 1478),
    ("bla_lesinit", 1489, 1545),
    ("bla_prhs", 1562, 1569),
    ("bla_pxinit", 1622, 1662),
    ("bla_bflow", 1338, 1374),
    ("bla_ffun", 2166, 2175),
    ("bla_substep_time", 1796, 1797),
    ("bla_les", 1945, 2020),
    ("bla_boxshift", 1819, 1826),
    ("bla_xys", 2069, 2107),
    ("bla_nonlin", 2251, 2288),
    ("bla_cfl", 2349, 2351),
    ("bla_vart", 2355, 2380),
    ("bla_rkweights", 2384, 2397),
    ("bla_linear", 2433, 2475),
    ("bla_press", 2486, 2527),
    ("bla_itinc", 2598, 2598),
]

NOOP_STUBS = ("ctim", "wall_time", "fft_identify")
SMAG_MAX_POINTS = 2_000_000  # nx*ny*nz; larger oracle grids keep iiles_smag = 0
NTHREAD = 64  # compile-time thread slots (par.f nthread); the harness never runs more


def par_text(nx: int, ny: int, nz: int, nthread: int = NTHREAD, pressure: bool = False) -> str:
    with open(os.path.join(REF_BLA, "par.f")) as f:
        txt = f.read()
    txt, n1 = re.subn(r"parameter \(nx=\d+,ny=\d+,nz=\d+\)",
                      f"parameter (nx={nx},ny={ny},nz={nz})", txt)
    txt, n2 = re.subn(r"parameter \(nthread=\d+\)", f"parameter (nthread={nthread})", txt)
    txt, n3 = re.subn(r"parameter \(pressure=\d\)", f"parameter (pressure={1 if pressure else 0})", txt)
    if (n1, n2, n3) != (1, 1, 1):
        raise RuntimeError("par.f layout not recognised")
    return txt


def generate_c(nx: int, ny: int, nz: int, pressure: bool = False) -> str:
    sources = []
    for fn in UNIT_FILES:
        with open(os.path.join(REF_BLA, fn)) as f:
            sources.append((fn, f.read()))
    with open(os.path.join(REF_BLA, "bla.f")) as f:
        bla = f.read()
    if nx * ny * nz <= SMAG_MAX_POINTS:
        bla, n = re.subn(r"iiles_smag = iiles\*0", "iiles_smag = iiles*1", bla)
        if n != 1:
            raise RuntimeError("bla.f iiles_smag switch not recognised")
    sources.append(("bla.f", bla))
    return translate(sources, par_text(nx, ny, nz, pressure=pressure), defines={"OPENMP"},
                     main_ranges=MAIN_RANGES, stubs_noop=NOOP_STUBS,
                     skip_units=("fft_identify",), provided=("stopnow",))


def _dir(nx: int, ny: int, nz: int, fma: bool = False, pressure: bool = False) -> str:
    return os.path.join(OUT_ROOT, f"{nx}x{ny}x{nz}" + ("_fma" if fma else "") + ("_p" if pressure else ""))


def lib_path(nx: int, ny: int, nz: int, fma: bool = False, pressure: bool = False) -> str:
    return os.path.join(_dir(nx, ny, nz, fma, pressure), "libsimson_ref.so")


def build(nx: int, ny: int, nz: int, force: bool = False, verbose: bool = False, fma: bool = False,
          pressure: bool = False) -> str:
    """Translate + compile the reference for one grid; returns the .so path.

    fma=True builds a second copy with fused multiply-add contraction
    (-mfma -ffp-contract=fast): the same reference with roundoff-level
    different arithmetic, used to measure how far the reference agrees with
    itself."""
    out_dir = _dir(nx, ny, nz, fma, pressure)
    so = os.path.join(out_dir, "libsimson_ref.so")
    harness = os.path.join(HERE, "ref_harness.c")
    translator = os.path.join(HERE, "f77c.py")
    stamp = hashlib.sha256()
    for p in (harness, translator, __file__):
        with open(p, "rb") as f:
            stamp.update(f.read())
    stamp = stamp.hexdigest()[:16]
    stamp_file = os.path.join(out_dir, "stamp")
    if not force and os.path.exists(so) and os.path.exists(stamp_file):
        with open(stamp_file) as f:
            if f.read().strip() == stamp:
                return so
    if not os.path.isdir(REF_BLA):
        if os.path.exists(so):
            return so
        raise FileNotFoundError(f"reference sources not found at {REF_BLA} and no prebuilt {so}")
    os.makedirs(out_dir, exist_ok=True)
    csrc = generate_c(nx, ny, nz, pressure)
    gen = os.path.join(out_dir, "ref_gen.c")
    with open(gen, "w") as f:
        f.write(csrc)
    fp = ["-mfma", "-ffp-contract=fast"] if fma else ["-ffp-contract=off"]
    cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-w", "-std=gnu11",
           "-fno-fast-math"] + fp + ["-I", out_dir, "-o", so + ".tmp", harness, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(so + ".tmp", so)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    return so


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("grid", nargs="*", default=["48x65x48"], help="NXxNYxNZ")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for g in a.grid:
        nx, ny, nz = (int(v) for v in g.split("x"))
        print(build(nx, ny, nz, force=a.force, verbose=True))
