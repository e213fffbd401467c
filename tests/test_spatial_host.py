"""Host parts of the spatial channel, no GPU: the fringe function of the
library (sgpu_fringe_function) against the reference's bla/ffun.f run by the
oracle, bit for bit; the channel base flows against the reference's
bla/cbflow.f; the base flow read from a velocity field (bla/rbflow.f, which
the oracle cannot run: it reads a file) against a direct synthesis."""
import numpy as np
import pytest

from simson_b200.bla import SimsonError, base_flow, base_flow_from_fields, fringe_function


@pytest.mark.parametrize("nx,xl,fringe", [
    (16, 48.0, (-13.0, 0.0, 7.0, 3.0, 1.0)),     # the fringe at the end of the box
    (16, 48.0, (10.0, -20.0, 5.0, 4.0, 2.0)),    # across the box end (two ranges, fmax added)
    (32, 100.0, (-30.0, -5.0, 12.0, 4.0, 0.7)),
    (16, 48.0, (-24.0, 23.0, 20.0, 20.0, 1.5)),  # nearly the whole box
])
def test_fringe_function_matches_reference(nx, xl, fringe, need_ref):
    ny = {16: 17, 32: 33}[nx]  # grids the oracle is built for anyway
    need_ref(nx, ny, 16)
    from refsim import RefSim
    fs, fe, fr, ff, fm = fringe
    ref = RefSim(nx, ny, 16, 2000.0, xl, 2 * np.pi, 0.01, cflux=False)
    ref.set_spatial(4, fs, fe, fr, ff, fm)
    f1, f2 = ref.fringe()
    lam = fringe_function(3 * nx // 2, xl, fs, fe, fr, ff, fm)
    assert np.array_equal(lam[0::2], f1)
    assert np.array_equal(lam[1::2], f2)
    assert lam.max() > 0.0


def test_fringe_outside_the_box_is_rejected():
    with pytest.raises(SimsonError):
        fringe_function(24, 48.0, -13.0, 0.0, -7.0, 3.0, 1.0)  # negative rise distance
    with pytest.raises(SimsonError):
        fringe_function(23, 48.0, -13.0, 0.0, 7.0, 3.0, 1.0)   # odd nxp


@pytest.mark.parametrize("fltype", [4, 5])
def test_channel_base_flows_match_reference(fltype, need_ref):
    need_ref(16, 17, 16)
    from refsim import RefSim
    ref = RefSim(16, 17, 16, 2000.0, 48.0, 2 * np.pi, 0.01, cflux=False)
    ref.set_spatial(fltype, -13.0, 0.0, 7.0, 3.0, 1.0)
    r1, r2 = ref.base_flow()
    b1, b2 = base_flow(fltype, 17, 24)
    assert np.array_equal(b1[:, :, :12], r1[:, :, :12])
    assert np.array_equal(b2[:, :, :12], r2[:, :, :12])


def test_base_flow_from_fields_synthesis():
    nx, nyp, nz, nxp, xl = 16, 9, 8, 24, 48.0
    rng = np.random.default_rng(5)
    fields = []
    for _ in range(3):
        f = np.zeros((nz, nyp, nx // 2), complex)
        f[0] = rng.normal(size=(nyp, nx // 2)) + 1j * rng.normal(size=(nyp, nx // 2))
        f[1] = 7.0  # kz != 0 is not read
        fields.append(f)
    b1, b2 = base_flow_from_fields(*fields, nxp=nxp, u0low=0.25, w0low=-0.5)
    x = np.arange(nxp) * xl / nxp
    alfa = 2 * np.pi * np.arange(nx // 2) / xl
    for i, f in enumerate(fields):
        c = f[0].copy()
        if i == 0:
            c[:, 0] += 0.25 - c[-1, 0].real
        if i == 2:
            c[:, 0] += -0.5 - c[-1, 0].real
        phys = c[:, :1].real + 2.0 * np.real(c[:, 1:] @ np.exp(1j * np.outer(alfa[1:], x)))
        assert np.allclose(b1[i, :, :nxp // 2], phys[:, 0::2], atol=1e-12)
        assert np.allclose(b2[i, :, :nxp // 2], phys[:, 1::2], atol=1e-12)
    # the lower wall (y = -1, the last point) takes u0low and w0low as its x mean
    for i, want in ((0, 0.25), (2, -0.5)):
        wall = np.concatenate([b1[i, -1, :nxp // 2], b2[i, -1, :nxp // 2]])
        assert abs(wall.mean() - want) <= 1e-12
