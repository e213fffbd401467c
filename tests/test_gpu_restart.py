"""Checkpoint and restart through the reference's .u file: two steps, the
field written with the wdiscbl layout (simson_b200/ufile.py), read back into
a new context, prhs, two more steps -- against four uninterrupted steps.
The restart is exact in exact arithmetic (the first RK stage has b_1 = 0:
the partial right-hand sides are a function of u, rebuilt by prhs, and px
under constant flux is re-solved every stage); in FP64 the two runs differ
by the roundoff of rebuilding p_v, p_omega through prhs instead of the
pencil kernel: u, v, w within 1e-10 (oddball kz plane excluded: it holds
the last nonlinear term and is never read)."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

NX, NY, NZ, RE, XL, ZL, DT = 48, 65, 48, 4200.0, 4 * np.pi, 2 * np.pi, 0.01


def rel(a, b):
    keep = np.ones(a.shape[0], bool)
    keep[a.shape[0] // 2] = False
    return float(np.linalg.norm(a[keep] - b[keep]) / np.linalg.norm(b[keep]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_from_u_file(tmp_path, precision):
    from simson_b200.bla import Channel
    from simson_b200.ufile import read_u, write_u
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 5)

    def channel(fields):
        ch = Channel(NX, NY, NZ, RE, XL, ZL, DT, precision=precision)
        ch.set_velocity(*fields)
        ch.prhs()
        return ch

    ch = channel((u, v, w))
    try:
        ch.step(4)
        ref = ch.state(3)
    finally:
        ch.close()
    ch = channel((u, v, w))
    try:
        ch.step(2)
        write_u(tmp_path / "restart.u", ch.state(3), RE, XL, ZL, t=2 * DT)
    finally:
        ch.close()
    head, fields = read_u(tmp_path / "restart.u")
    assert head["t"] == 2 * DT and (head["nx"], head["nyp"], head["nzc"]) == (NX, NY, NZ)
    ch = channel(fields)
    try:
        ch.step(2)
        got = ch.state(3)
    finally:
        ch.close()
    tol = 1e-10 if precision == "fp64" else 1e-5
    errs = [rel(got[k], ref[k]) for k in range(3)]
    print(precision, "restart vs continuous:", ["%.1e" % e for e in errs])
    assert max(errs) <= tol, errs
