"""Spatial channel (bla.i spat = .true., spatially developing Poiseuille flow,
fltype 4, ibc = 0): the fringe forcing of bla/fring.f in step 2 and in the
pressure (bla/fringp.f), against the reference run the same way (its own
bflow for the base flow, ffun before every substep, px = 0 and no constant
flux).  Tolerances as the temporal channel's: relative L2 1e-11 on u, v, w
together and 1e-10 per slot (FP64), 1e-5 between the mixed path and FP64."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 33, 16
RE, XL, ZL, DT = 2000.0, 48.0, 2 * np.pi, 0.02
FRINGE = dict(fstart=-13.0, fend=0.0, frise=7.0, ffall=3.0, fmax=1.0)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _gpu(nx, ny, nz, precision, fringe=True, nst=3, dt=DT):
    from simson_b200.bla import Channel, base_flow
    ch = Channel(nx, ny, nz, RE, XL, ZL, dt, cflux=False, px=0.0, precision=precision, nst=nst)
    if fringe:
        ch.set_base_flow(*base_flow(4, ny, 3 * nx // 2))
        ch.set_fringe(**FRINGE)
    return ch


def _ref(nx, ny, nz, nst=3, dt=DT, pressure=False):
    from refsim import RefSim
    r = RefSim(nx, ny, nz, RE, XL, ZL, dt, cflux=False, nst=nst, pressure=pressure)
    r.set_spatial(4, **FRINGE)
    return r


def test_spatial_channel_ten_steps_vs_reference(need_ref):
    need_ref(NX, NY, NZ)
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 21)
    ref = _ref(NX, NY, NZ)
    ref.set_velocity(u, v, w)
    ref.start()
    ref.step(10)
    gpu = _gpu(NX, NY, NZ, "fp64")
    try:
        gpu.set_velocity(u, v, w)
        gpu.start()
        gpu.step(10)
        gs, sc = gpu.state(), gpu.scalars()
    finally:
        gpu.close()
    rs, rsc = ref.state(), ref.scalars()
    uvw = rel(np.concatenate([gs[k].ravel() for k in range(3)]), np.concatenate([rs[k].ravel() for k in range(3)]))
    per = [rel(gs[k], rs[k]) for k in range(7)]
    print("spatial channel, 10 steps: u,v,w %.2e" % uvw, ["%.1e" % e for e in per])
    assert uvw <= 1e-11
    assert max(per) <= 1e-10
    assert sc["px"] == 0.0 and rsc["px"] == 0.0
    assert abs(sc["t"] - rsc["t"]) <= 1e-12
    # the fringe does something: without it the state differs at O(dt fmax)
    gpu = _gpu(NX, NY, NZ, "fp64", fringe=False)
    try:
        gpu.set_velocity(u, v, w)
        gpu.start()
        gpu.step(10)
        nf = gpu.state(3)
    finally:
        gpu.close()
    assert rel(nf[0], rs[0]) > 1e-4


def test_spatial_channel_rk4_variable_dt_vs_reference(need_ref):
    """nst = 4 with the variable time step (dt <= 0 in bla.i): the CFL rule
    of bla/bla.f:2355-2380, bounded by the fringe's limit 1.96/fmax."""
    need_ref(NX, NY, NZ)
    from simson_b200.driver import next_dt
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 22)
    cflmax = 0.8 * np.sqrt(8.0)
    dtmax = 1.96 / FRINGE["fmax"]
    from refsim import RefSim
    ref = RefSim(NX, NY, NZ, RE, XL, ZL, -dtmax, cflux=False, nst=4, cflmaxin=0.8)
    ref.set_spatial(4, **FRINGE)
    ref.set_velocity(u, v, w)
    ref.start()
    ref.step(6)
    gpu = _gpu(NX, NY, NZ, "fp64", nst=4, dt=1.0)
    try:
        gpu.set_velocity(u, v, w)
        dtn = min(cflmax / gpu.cfl_rate(), dtmax)
        gpu.set_dt(dtn)
        gpu.start()
        t = 0.0
        for _ in range(6):
            gpu.substeps(3)
            sc = gpu.scalars()
            dtnp1 = next_dt(dtn, sc["cfl"], cflmax, dtmax, t, 1.0e30, 0.0)
            gpu.set_dt(dtnp1)
            gpu.substeps(1)
            t += dtn
            dtn = dtnp1
        gs, sc = gpu.state(), gpu.scalars()
    finally:
        gpu.close()
    rs, rsc = ref.state(), ref.scalars()
    uvw = rel(np.concatenate([gs[k].ravel() for k in range(3)]), np.concatenate([rs[k].ravel() for k in range(3)]))
    print("spatial channel, RK4 variable dt, 6 steps: u,v,w %.2e, t %.15g vs %.15g" % (uvw, sc["t"], rsc["t"]))
    assert uvw <= 1e-10
    assert abs(sc["t"] - rsc["t"]) <= 1e-12 * rsc["t"]


def test_spatial_channel_mixed_vs_fp64():
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 21)
    out = []
    for prec in ("fp64", "mixed"):
        ch = _gpu(NX, NY, NZ, prec)
        try:
            ch.set_velocity(u, v, w)
            ch.start()
            ch.step(20)
            out.append(ch.state(3))
        finally:
            ch.close()
    keep = np.ones(NZ, bool)
    keep[NZ // 2] = False  # the oddball plane, as the other mixed-precision gates
    errs = [rel(out[1][k][keep], out[0][k][keep]) for k in range(3)]
    print("spatial channel, mixed vs FP64 after 20 steps:", ["%.1e" % e for e in errs])
    assert max(errs) <= 1e-5


def test_spatial_pressure_vs_reference(need_ref):
    """The pressure of a spatial run includes the fringe force (bla/fringp.f)."""
    nx, ny, nz = 16, 17, 16
    from build_ref import REF_BLA, lib_path
    import os
    if not (os.path.isdir(REF_BLA) or os.path.exists(lib_path(nx, ny, nz, pressure=True))):
        pytest.skip("pressure variant of the oracle neither buildable nor prebuilt")
    u, v, w = channel_field(nx, ny, nz, XL, ZL, 0.05, 23)
    ref = _ref(nx, ny, nz, pressure=True)
    ref.set_velocity(u, v, w)
    ref.start()
    ref.step(2)
    state = ref.state()
    rp = ref.pressure()
    gpu = _gpu(nx, ny, nz, "fp64")
    try:
        gpu.set_state(state)
        gp = gpu.pressure()
        gpu.set_fringe(0.0, 0.0, 1.0, 1.0, 0.0)
        gp0 = gpu.pressure()
    finally:
        gpu.close()
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    e = rel(gp[keep], rp[keep])
    print("spatial pressure vs reference: %.2e (without the fringe term %.2e)" % (e, rel(gp0[keep], rp[keep])))
    assert e <= 1e-10
    assert rel(gp0[keep], rp[keep]) > 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spatial_shards_and_graphs_equal_one_direct_context(precision):
    """The fringe under the multi-GPU decomposition (two shard contexts,
    emulated on one device: each applies the fringe on its own xz-planes) and
    under CUDA-graph replay (the fringe is part of the captured launch
    pattern) gives the state of one context launching directly, bit for bit."""
    import os
    from simson_b200.shard import LocalShards
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 24)

    def make():
        ch = _gpu(NX, NY, NZ, precision)
        ch.set_velocity(u, v, w)
        ch.prhs()
        return ch

    old = os.environ.get("SIMSON_GRAPHS")
    os.environ["SIMSON_GRAPHS"] = "0"
    try:
        one = make()
    finally:
        if old is None:
            os.environ.pop("SIMSON_GRAPHS")
        else:
            os.environ["SIMSON_GRAPHS"] = old
    try:
        one.step(3)
        ref = one.state(7)
    finally:
        one.close()
    graph = make()
    try:
        graph.step(3)
        got_graph = graph.state(7)
    finally:
        graph.close()
    sh = LocalShards(make, 2, "cuda:0")
    try:
        sh.step(3)
        got_sh = sh.state(7)
    finally:
        sh.close()
    for k in range(7):
        assert np.array_equal(got_graph[k], ref[k]), k
        assert np.array_equal(got_sh[k], ref[k]), k
