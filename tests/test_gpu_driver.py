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
