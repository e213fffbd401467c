"""The bla.i-driven host (simson_b200.driver) end to end on the GPU against
the reference run with the same deck values: a deck in the form of the
reference's channel example (4-stage RK, variable time step from the CFL
number, amp.stat every two steps, one intermediate save), an initial .u
written by simson_b200.ufile, and the translated reference stepping the
same field with nst = 4 and its own variable-step rule (getdt, then
bla/bla.f:2355-2380).  Gates: the final field (end.u) within 1e-10 of the
reference's (u, v, w relative L2), the time reached and the last time step
to 1e-12; the 4-stage scheme with a fixed step as well."""
import os

import numpy as np
import pytest

from deck import bla_i
from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

NX, NY, NZ, XL, ZL, RE = 48, 65, 48, 4 * np.pi, 2 * np.pi, 4200.0


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_deck(tmp_path, **kw):
    from simson_b200 import ufile
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 8)
    ufile.write_u(str(tmp_path / "init.u"), [u, v, w], RE, XL, ZL, 0.0)
    (tmp_path / "bla.i").write_text(bla_i(xl=XL, **kw))
    return (u, v, w)


def reference(uvw, steps, dt, nst):
    from refsim import RefSim
    ref = RefSim(NX, NY, NZ, RE, XL, ZL, dt, nst=nst, cflmaxin=0.8)
    ref.set_velocity(*uvw)
    ref.start()
    ref.step(steps)
    return ref.state()[:3], ref.scalars()


@pytest.mark.parametrize("dt", [0.0, 0.01])
def test_driver_four_stage_channel_deck(tmp_path, need_ref, dt):
    from simson_b200 import driver, ufile
    need_ref(NX, NY, NZ)
    steps = 6
    uvw = make_deck(tmp_path, dt=dt, nst=4, maxit=4 * steps, icfl=4, iamp=8, saves=((0.025, "t1.u"),))
    res = driver.run(str(tmp_path), log=lambda *a: None)
    assert res["steps"] == steps
    head, got = ufile.read_u(str(tmp_path / "end.u"))
    want, sc = reference(uvw, steps, dt, 4)
    errs = [rel(got[k], want[k]) for k in range(3)]
    print("driver dt", dt, "vs reference:", ["%.2e" % e for e in errs], "t %.15f / %.15f" % (head["t"], sc["t"]),
          "dt %.15f / %.15f" % (res["dt"], sc["dtn"]))
    assert max(errs) <= 1e-10, errs
    assert abs(head["t"] - sc["t"]) <= 1e-12 * max(1.0, sc["t"])
    assert abs(res["dt"] - sc["dtn"]) <= 1e-12 * sc["dtn"]
    lines = (tmp_path / "amp.stat").read_text().splitlines()
    assert len(lines) == steps // 2 and all(len(ln.split()) == 19 for ln in lines)
    assert os.path.exists(tmp_path / "t1.u")


SX, SY, SZ, SXL, SRE = 32, 33, 16, 48.0, 2000.0
FR = (1.0, -13.0, 0.0, 7.0, 3.0)  # fmax, fstart, fend, frise, ffall


@pytest.mark.parametrize("rbfl", [False, True])
def test_driver_spatial_channel_deck(tmp_path, need_ref, rbfl):
    """A spatial deck (spat, the fringe of the reference's spatial-channel
    example, fltype 4 in the initial field, cflux off, RK4 with the variable
    time step under the fringe's bound 1.96/fmax), the base flow computed or
    read from a file (rbfl), against the reference run with its own bflow and
    ffun."""
    from refsim import RefSim
    from simson_b200 import driver, ufile
    need_ref(SX, SY, SZ)
    steps = 6
    u, v, w = channel_field(SX, SY, SZ, SXL, ZL, 0.05, 31)
    ufile.write_u(str(tmp_path / "init.u"), [u, v, w], SRE, SXL, ZL, 0.0, fltype=4)
    if rbfl:  # the Poiseuille base flow as a field file
        y = np.cos(np.pi * np.arange(SY) / (SY - 1))
        b = np.zeros((SZ, SY, SX // 2), complex)
        b[0, :, 0] = 1.0 - y ** 2
        ufile.write_u(str(tmp_path / "baseflow.u"), [b, 0 * b, 0 * b], SRE, SXL, ZL, 0.0, fltype=4)
    (tmp_path / "bla.i").write_text(bla_i(xl=SXL, dt=0.0, nst=4, maxit=4 * steps, icfl=4, cflux=False, retau=0.0,
                                          spat=True, rbfl="baseflow.u" if rbfl else None, fringe=FR))
    res = driver.run(str(tmp_path), log=lambda *a: None)
    assert res["steps"] == steps and res["px"] == 0.0
    head, got = ufile.read_u(str(tmp_path / "end.u"))
    ref = RefSim(SX, SY, SZ, SRE, SXL, ZL, -1.96 / FR[0], cflux=False, nst=4, cflmaxin=0.8)
    ref.set_spatial(4, FR[1], FR[2], FR[3], FR[4], FR[0])
    ref.set_velocity(u, v, w)
    ref.start()
    ref.step(steps)
    want, sc = ref.state()[:3], ref.scalars()
    errs = [rel(got[k], want[k]) for k in range(3)]
    print("spatial driver (rbfl %s) vs reference:" % rbfl, ["%.2e" % e for e in errs],
          "t %.15f / %.15f" % (head["t"], sc["t"]))
    assert max(errs) <= 1e-10, errs
    assert abs(head["t"] - sc["t"]) <= 1e-12 * max(1.0, sc["t"])
    assert abs(res["dt"] - sc["dtn"]) <= 1e-12 * sc["dtn"]
