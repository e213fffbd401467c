"""ADM-RT large-eddy model on the device against the translated reference
(iles = 1, sgs.i of the reference's LES example: cut-off 1/1.5, N = 5,
chi = 0.2, tensorial filtering unless stated).

The seeded fields carry modes up to |k| = nx/2 - 2 so that the high pass is
not empty.  gu is a linear filter of u, and a smooth part of u passes it to
roundoff only, so its error is measured relative to the velocity it was
filtered from: within 1e-12 after the start-up prhs, 1e-10 after substeps.
The state keeps the channel step's gate: u, v, w within 1e-11 and every other
field within 1e-10 (relative L2).  gu of the oddball plane (kz = -nz/2) is
left out: linearbl never visits that plane and step 2 never reads it."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _pair(nx, ny, nz, xl, zl, re, dt, rms, seed, need_ref, **les):
    need_ref(nx, ny, nz)
    from refsim import RefSim
    from simson_b200.bla import Channel
    u, v, w = channel_field(nx, ny, nz, xl, zl, rms, seed, kmax=min(nx, nz) // 2 - 2)
    ref = RefSim(nx, ny, nz, re, xl, zl, dt)
    ref.set_les(**les)
    ref.set_velocity(u, v, w)
    ref.start()
    gpu = Channel(nx, ny, nz, re, xl, zl, dt)
    gpu.set_les(**les)
    gpu.set_velocity(u, v, w)
    gpu.start()
    return ref, gpu


def _gu_errors(ref, gpu, nz):
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    g = gpu.les_gu()
    rs = ref.state()
    return [float(np.linalg.norm(g[c][keep] - ref.gu(c + 1)[keep]) / np.linalg.norm(rs[c][keep])) for c in range(3)]


def _state_errors(ref, gpu):
    rs, gs = ref.state(), gpu.state()
    return [rel_l2(gs[k], rs[k]) for k in range(7)]


@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_les_start_matches_reference(grid, need_ref):
    nx, ny, nz = grid
    ref, gpu = _pair(nx, ny, nz, 4 * np.pi, 2 * np.pi, 4200.0, 0.01, 0.05, 3, need_ref)
    errs = _gu_errors(ref, gpu, nz)
    assert max(errs) < 1e-12, errs


@pytest.mark.parametrize("mode", [2, 1, 0])
def test_les_substeps_match_reference(mode, need_ref):
    nx, ny, nz = 16, 17, 16
    ref, gpu = _pair(nx, ny, nz, 4 * np.pi, 2 * np.pi, 4200.0, 0.01, 0.05, 5, need_ref, ihighorder=mode)
    for _ in range(6):
        ref.substep()
        gpu.substep()
        e = _state_errors(ref, gpu)
        assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e
        g = _gu_errors(ref, gpu, nz)
        assert max(g) < 1e-10, g


def test_les_config_d_ten_steps(need_ref):
    """The LES configuration: 64x97x64 on 2pi x 2 x pi, Re 4200, rms 0.1,
    dt 0.005, ten RK3 steps with ADM-RT."""
    nx, ny, nz = 64, 97, 64
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 4, need_ref)
    for _ in range(30):
        ref.substep()
        gpu.substep()
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e
    assert max(_gu_errors(ref, gpu, nz)) < 1e-10


def test_les_relaxation_acts():
    """chi > 0 removes energy at the smallest scales: after 20 steps the
    high-pass energy with the model is below the one without it."""
    from simson_b200.bla import Channel
    nx, ny, nz = 48, 65, 48
    xl, zl = 2 * np.pi, np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 8, kmax=20)
    e = {}
    for chi in (0.0, 5.0):
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005)
        ch.set_les(chi=chi)
        ch.set_velocity(u, v, w)
        ch.start()
        ch.substeps(60)
        g = ch.les_gu()
        g[:, :, :, 0] = 0.0  # kx = 0 column carries the mean profile's high pass
        e[chi] = float(np.sum(np.abs(g) ** 2))
        ch.close()
    assert e[5.0] < 0.9 * e[0.0], e


def test_les_mixed_close_to_fp64():
    from simson_b200.bla import FP64, MIXED, Channel
    nx, ny, nz = 64, 97, 64
    xl, zl = 2 * np.pi, np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 4, kmax=30)
    out = {}
    for prec in (FP64, MIXED):
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005, precision=prec)
        ch.set_les()
        ch.set_velocity(u, v, w)
        ch.start()
        ch.substeps(60)
        out[prec] = ch.state(3)
        ch.close()
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    err = rel_l2(np.stack(out[MIXED])[:, keep], np.stack(out[FP64])[:, keep])
    assert err < 1e-5, err


# --- eddy-viscosity model (iles = 2, dynamic Smagorinsky) -------------------

def _tau_errors(ref, gpu, nz):
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    t = gpu.sgs_stress()
    out = []
    for c in range(6):
        r = ref.tau(c + 1)
        out.append(float(np.linalg.norm(t[c][keep] - r[keep]) / max(np.linalg.norm(r[keep]), 1e-300)))
    return out


@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_dynamic_smagorinsky_stress_matches_reference(grid, need_ref):
    """tau_ij of les.f and sigma_i of sgs_stress.f on the start-up state
    (evaluated inside the first substep), then the state after it."""
    nx, ny, nz = grid
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 6, need_ref, iles=2)
    ref.substep()
    gpu.substep()
    te = _tau_errors(ref, gpu, nz)
    assert max(te) < 1e-11, te
    se = _gu_errors(ref, gpu, nz)
    assert max(se) < 1e-11, se
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e


def test_dynamic_smagorinsky_substeps(need_ref):
    nx, ny, nz = 16, 17, 16
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 7, need_ref, iles=2)
    for _ in range(6):
        ref.substep()
        gpu.substep()
        e = _state_errors(ref, gpu)
        assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e


def test_dynamic_smagorinsky_config_d(need_ref):
    """The LES configuration 64x97x64, 2pi x 2 x pi, ten RK3 steps."""
    nx, ny, nz = 64, 97, 64
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 4, need_ref, iles=2)
    for _ in range(30):
        ref.substep()
        gpu.substep()
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e
    assert max(_tau_errors(ref, gpu, nz)) < 1e-10


@pytest.mark.parametrize("cs,ineg", [(0.1, 1), (0.0, 0), (0.0, 2)])
def test_smagorinsky_variants(cs, ineg, need_ref):
    """Fixed Smagorinsky constant, and the dynamic model without clipping and
    with the nu_t + nu >= 0 clip."""
    nx, ny, nz = 16, 17, 16
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 8, need_ref, iles=2, cs=cs, ineg=ineg)
    for _ in range(3):
        ref.substep()
        gpu.substep()
    assert max(_tau_errors(ref, gpu, nz)) < 1e-10
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e


# --- HPF eddy-viscosity model (iles = 3, fixed constant) --------------------

@pytest.mark.parametrize("grid", [(16, 17, 16), (48, 65, 48)])
def test_hpf_smagorinsky_matches_reference(grid, need_ref):
    """tau_ij = -2 cs^2 Delta^2 |S(H u)| S(H u) of bla/les.f:883-966, 1515 on
    the high-pass filtered velocities and vorticities of bla/linearbl.f:
    1871-2060 (prhs.f at the start), its divergence sigma, the state."""
    nx, ny, nz = grid
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 9, need_ref, iles=3, cs=0.12)
    assert max(_gu_errors(ref, gpu, nz)) < 1e-12  # H u, v, w after the start-up
    ref.substep()
    gpu.substep()
    te = _tau_errors(ref, gpu, nz)
    assert max(te) < 1e-11, te
    se = _gu_errors(ref, gpu, nz)  # sigma
    assert max(se) < 1e-11, se
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e


@pytest.mark.parametrize("ihighorder", [0, 1, 2])
def test_hpf_smagorinsky_substeps(ihighorder, need_ref):
    nx, ny, nz = 16, 17, 16
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 10, need_ref, iles=3, cs=0.1,
                     ihighorder=ihighorder)
    for _ in range(6):
        ref.substep()
        gpu.substep()
        e = _state_errors(ref, gpu)
        assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e
    assert max(_tau_errors(ref, gpu, nz)) < 1e-10


def test_hpf_smagorinsky_config_d(need_ref):
    """The LES configuration 64x97x64, ten RK3 steps."""
    nx, ny, nz = 64, 97, 64
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 11, need_ref, iles=3, cs=0.1)
    for _ in range(30):
        ref.substep()
        gpu.substep()
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e


@pytest.mark.parametrize("grid,ineg", [((16, 17, 16), 1), ((48, 65, 48), 1), ((16, 17, 16), 0), ((16, 17, 16), 2)])
def test_dynamic_hpf_matches_reference(grid, ineg, need_ref):
    """The dynamic HPF procedure (cs = 0): L_ij of the resolved velocity, M_ij
    of the primary and the test-filtered secondary high-pass strain, the
    clipped coefficient, tau = -2 C Delta^2 |S(H u)| S(H u).  tau and sigma
    are compared after the step-2 half of the first substep: the reference's
    step 3 then writes the secondary filtered fields into taur slots 1-5
    (bla/linearbl.f:2067-2250); the state after six substeps."""
    nx, ny, nz = grid
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 12, need_ref, iles=3, cs=0.0, ineg=ineg)
    ref.nonlin_only()
    gpu.nonlinbl()
    te = _tau_errors(ref, gpu, nz)
    assert max(te) < 1e-11, te
    assert max(_gu_errors(ref, gpu, nz)) < 1e-11
    ref.linear_only()
    gpu.linearbl()
    for _ in range(5):
        ref.substep()
        gpu.substep()
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e


def test_dynamic_hpf_config_d(need_ref):
    """The LES configuration 64x97x64, ten RK3 steps of the dynamic HPF model."""
    nx, ny, nz = 64, 97, 64
    ref, gpu = _pair(nx, ny, nz, 2 * np.pi, np.pi, 4200.0, 0.005, 0.1, 13, need_ref, iles=3, cs=0.0)
    for _ in range(30):
        ref.substep()
        gpu.substep()
    e = _state_errors(ref, gpu)
    assert max(e[:3]) < 1e-11 and max(e) < 1e-10, e
    # taur slot 6 (tau_33) is the only one the reference's step 3 leaves
    assert _tau_errors(ref, gpu, nz)[5] < 1e-10


def test_dynamic_hpf_mixed_close_to_fp64():
    from simson_b200.bla import Channel
    nx, ny, nz = 48, 65, 48
    u, v, w = channel_field(nx, ny, nz, 2 * np.pi, np.pi, 0.1, 14, kmax=min(nx, nz) // 2 - 2)
    out = []
    for prec in ("fp64", "mixed"):
        ch = Channel(nx, ny, nz, 4200.0, 2 * np.pi, np.pi, 0.005, precision=prec)
        try:
            ch.set_les(iles=3, cs=0.0)
            ch.set_velocity(u, v, w)
            ch.start()
            ch.step(10)
            out.append(ch.state(3))
        finally:
            ch.close()
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    errs = [rel_l2(out[1][k][keep], out[0][k][keep]) for k in range(3)]
    assert max(errs) < 1e-5, errs
