"""The C ABI without a GPU: the library loads, and every function that
include/simson_b200.h declares is exported by it (the entry points a Fortran
or C host binds to).  No compute call is made."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "simson_b200.h")


def declared():
    with open(HEADER) as f:
        txt = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    return sorted(set(re.findall(r"\b(sgpu_\w+)\s*\(", txt)))


def test_header_declares_the_step_and_its_neighbours():
    names = declared()
    for must in ("sgpu_init", "sgpu_prhs", "sgpu_nonlin", "sgpu_linear", "sgpu_step_rk", "sgpu_upload_state",
                 "sgpu_download_state", "sgpu_amplitudes", "sgpu_xys_sample", "sgpu_set_les", "sgpu_set_shard",
                 "sgpu_copy_block", "sgpu_offload_steps", "sgpu_pressure", "sgpu_box_filter_sample",
                 "sgpu_xys_get", "sgpu_xys_reset", "sgpu_finalize", "sgpu_nonlin_noalloc"):
        assert must in names


def test_library_exports_every_declared_function():
    from simson_b200 import build
    lib = ctypes.CDLL(build.build())
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


SGPU_E_PARAM = -1


def _lib():
    from simson_b200 import build
    from simson_b200.bla import load_library
    build.build()
    return load_library(build=False)


def test_init_rejects_invalid_parameters():
    """sgpu_init validates the grid and the run parameters before it touches
    the device (nx a multiple of 4, nz even, ny odd and >= 9, nst = 3,
    dt, Re and box lengths positive, a known precision)."""
    from simson_b200.bla import SgpuParams
    lib = _lib()
    good = dict(nx=48, ny=65, nz=48, re=4200.0, xl=12.566, zl=6.283, dt=0.01, nst=3, cflux=1, mflux=4.0 / 3.0,
                px=-2.0 / 4200.0, rot=0.0, icfl=3, precision=0, device=0)
    bad = [dict(nx=46), dict(nx=0), dict(nz=47), dict(ny=64), dict(ny=7), dict(nst=2), dict(nst=5), dict(dt=0.0), dict(dt=-1.0),
           dict(re=0.0), dict(xl=0.0), dict(zl=-1.0), dict(precision=2), dict(dt=float("nan"))]
    for change in bad:
        p = SgpuParams(**{**good, **change})
        ctx = ctypes.c_void_p(1)
        rc = lib.sgpu_init(ctypes.byref(p), ctypes.byref(ctx))
        assert rc == SGPU_E_PARAM, change
        assert not ctx.value, change
    assert lib.sgpu_init(None, None) == SGPU_E_PARAM


def test_entry_points_reject_a_null_context():
    lib = _lib()
    dp = ctypes.POINTER(ctypes.c_double)
    buf = (ctypes.c_double * 16)()
    p = ctypes.cast(buf, dp)
    assert lib.sgpu_prhs(None) == SGPU_E_PARAM
    assert lib.sgpu_nonlin(None) == SGPU_E_PARAM
    assert lib.sgpu_linear(None) == SGPU_E_PARAM
    assert lib.sgpu_step_rk(None, 3) == SGPU_E_PARAM
    assert lib.sgpu_offload_steps(None, p, p, 1) == SGPU_E_PARAM
    assert lib.sgpu_amplitudes(None, p, p) == SGPU_E_PARAM
    assert lib.sgpu_xys_sample(None, ctypes.c_double(0.01)) == SGPU_E_PARAM
    assert lib.sgpu_xys_get(None, p, p) == SGPU_E_PARAM
    assert lib.sgpu_xys_reset(None) == SGPU_E_PARAM
    assert lib.sgpu_set_shard(None, 0, 1, 0, 1) == SGPU_E_PARAM
    assert lib.sgpu_finalize(None) == 0
    for rc in (0, -1, -2, -3, -4, -5):
        assert lib.sgpu_error_string(rc)


def test_nonlin_noalloc_rejects_invalid_arguments():
    """The allocation-free step 2 checks its arguments before it touches the
    device: null pointers, an invalid grid and a precision other than FP64
    (its arrays are complex doubles) come back as SGPU_E_PARAM."""
    from simson_b200.bla import SgpuParams
    lib = _lib()
    lib.sgpu_nonlin_noalloc.argtypes = [ctypes.POINTER(SgpuParams), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    good = dict(nx=48, ny=65, nz=48, re=4200.0, xl=12.566, zl=6.283, dt=0.01, nst=3, cflux=1, mflux=4.0 / 3.0,
                px=-2.0 / 4200.0, rot=0.0, icfl=3, precision=0, device=0)
    buf = ctypes.c_void_p(16)  # never dereferenced: every case below is rejected first
    p = SgpuParams(**good)
    assert lib.sgpu_nonlin_noalloc(None, buf, buf, None, None) == SGPU_E_PARAM
    assert lib.sgpu_nonlin_noalloc(ctypes.byref(p), None, buf, None, None) == SGPU_E_PARAM
    assert lib.sgpu_nonlin_noalloc(ctypes.byref(p), buf, None, None, None) == SGPU_E_PARAM
    for change in (dict(nx=46), dict(nx=0), dict(ny=64), dict(ny=7), dict(nz=47), dict(xl=0.0), dict(precision=1)):
        q = SgpuParams(**{**good, **change})
        assert lib.sgpu_nonlin_noalloc(ctypes.byref(q), buf, buf, None, None) == SGPU_E_PARAM, change


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++11")])
def test_header_compiles_on_its_own(tmp_path, lang, std):
    """A C or C++ host includes the header first: it must bring what it uses."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / "host.txt"
    src.write_text('#include "simson_b200.h"\nint main(void) { return 0; }\n')
    r = subprocess.run([cc, "-std=" + std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                        os.path.join(ROOT, "include"), "-x", lang, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

