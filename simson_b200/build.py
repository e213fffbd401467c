"""Build the CUDA library in-tree: simson_b200/_lib/libsimson_b200.so (sm_100a).

The library is the product's C ABI (include/simson_b200.h); Python reaches it
through ctypes (simson_b200/bla.py), a Fortran host through ISO_C_BINDING.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libsimson_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "simson.cu"), os.path.join(HERE, "csrc", "noalloc.cu"),
           os.path.join(HERE, "csrc", "mixed.cu")]
# units built with fused multiply-add contraction (the mixed-precision path)
FMAD_SOURCES = {os.path.join(HERE, "csrc", "mixed.cu")}
DEPS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + [
    os.path.join(ROOT, "include", "simson_b200.h")]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS + [__file__])


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    # The FP64 path is built without FMA contraction: the reference's
    # arithmetic (gfortran/gcc for x86-64) rounds every product, and the stiff
    # tau solves (lambda ~ 1e6) amplify the difference between fused and
    # separate rounding to ~1e-12.  Set SIMSON_FMAD=1 to allow contraction.
    # The mixed-precision unit is built with contraction (it is checked
    # against the FP64 path at 1e-5, not bit for bit).
    fmad_all = os.environ.get("SIMSON_FMAD") == "1"
    objs = []
    procs = []
    for src in SOURCES:
        fmad = "true" if (fmad_all or src in FMAD_SOURCES) else "false"
        obj = os.path.join(LIB_DIR, os.path.splitext(os.path.basename(src))[0] + ".o")
        cmd = [nvcc(), ARCH, "-O3", "-lineinfo", "-std=c++17", f"-fmad={fmad}", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    if any(p.wait() != 0 for p in procs):
        raise subprocess.CalledProcessError(1, "nvcc")
    cmd = [nvcc(), ARCH, "-shared", "-o", LIB + ".tmp"] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    os.replace(LIB + ".tmp", LIB)
    return LIB


HOSTCHECK = os.path.join(LIB_DIR, "libsimson_hostcheck.so")


def build_hostcheck(force: bool = False) -> str:
    """Host (CPU) build of the step-3 pencil algebra for the CPU unit tests."""
    src = os.path.join(HERE, "csrc", "hostcheck.cu")
    if not force and os.path.exists(HOSTCHECK) and all(
            os.path.getmtime(d) <= os.path.getmtime(HOSTCHECK) for d in DEPS + [__file__]):
        return HOSTCHECK
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc(), ARCH, "-O2", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
           "--expt-relaxed-constexpr", "-o", HOSTCHECK + ".tmp", src]
    subprocess.run(cmd, check=True)
    os.replace(HOSTCHECK + ".tmp", HOSTCHECK)
    return HOSTCHECK


if __name__ == "__main__":
    print(build(force=True, verbose=True))
    print(build_hostcheck(force=True))
