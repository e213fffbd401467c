"""The C ABI without a GPU: the library loads, and every function that
include/simson_b200.h declares is exported by it (the entry points a Fortran
or C host binds to).  No compute call is made."""
import ctypes
import os
import re

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
                 "sgpu_copy_block", "sgpu_offload_steps", "sgpu_finalize"):
        assert must in names


def test_library_exports_every_declared_function():
    from simson_b200 import build
    lib = ctypes.CDLL(build.build())
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
