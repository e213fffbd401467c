"""Mixed precision (FP32 FFTs, products, Chebyshev transforms and
velocity/vorticity storage; FP64 tau solves, mean flow and partial RHS)
against the FP64 path on the same seeded field.  Gate: relative L2 on
u, v, w <= 1e-5 after 100 steps."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


def rel(a, b):
    """Relative L2 over the modes the dynamics uses: the oddball plane
    kz = -nz/2 of u, v, w holds the last nonlinear term (the reference leaves
    it there too, bla/linearbl.f skips that plane) and is zeroed by every
    reader (bla/getxz.f), so it is left out."""
    nz = a.shape[0]
    keep = np.ones(nz, bool)
    keep[nz // 2] = False
    a, b = a[keep], b[keep]
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("grid,rms,steps", [((48, 65, 48), 0.02, 100), ((64, 97, 64), 0.1, 100)])
def test_mixed_vs_fp64(grid, rms, steps):
    from simson_b200.bla import FP64, MIXED, Channel
    nx, ny, nz = grid
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, rms, 4)
    out = []
    for prec in (FP64, MIXED):
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01 if rms < 0.05 else 0.005, precision=prec)
        ch.set_velocity(u, v, w)
        ch.prhs()
        ch.step(steps)
        out.append((ch.state(3), ch.scalars()))
        ch.close()
    (s64, c64), (s32, c32) = out
    errs = [rel(s32[k], s64[k]) for k in range(3)]
    print(grid, "mixed vs fp64 after", steps, "steps:", ["%.2e" % e for e in errs], "px", c32["px"], c64["px"])
    assert max(errs) <= 1e-5, errs
    assert np.isfinite(c32["cfl"]) and abs(c32["cfl"] - c64["cfl"]) <= 1e-5 * c64["cfl"]


@pytest.mark.slow
def test_wall_shear_config_b_2000_steps():
    """Configuration B (192x129x160, 4pi x 2 x 2pi, Re 4200, dt 0.005, rms
    0.1): after 2000 RK3 steps the mixed-precision path's wall shear, Re_tau
    (h+) and bulk Reynolds number stay within 0.5 % of the FP64 path's
    (amp.stat quantities, bla/wampbl.f)."""
    from simson_b200.bla import FP64, MIXED, Channel
    nx, ny, nz = 192, 129, 160
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.1, 2)
    rows = {}
    for prec in (FP64, MIXED):
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005, precision=prec)
        ch.set_velocity(u, v, w)
        ch.start()
        ch.step(2000)
        _, rows[prec] = ch.amplitudes()
        ch.close()
    for k in ("tau1", "tau2", "hplus", "re_bulk"):
        a, b = rows[MIXED][k], rows[FP64][k]
        assert abs(a - b) <= 5e-3 * abs(b), (k, a, b)
