"""Failure detection of the tensor-core kernels without a GPU fault: every
mbarrier wait of the mixed path's Chebyshev GEMM (k_cheb_tc) and of the
learned SGS model (k_sgs_mlp) is bounded.  sgpu_set_wait_limit(limit,
test_timeout=1) makes the first wait of each launch wait on a barrier that
nothing completes, with a short limit; the kernel must then let its own
copies and MMAs finish, free its tensor memory and return, the host must
read SGPU_E_TIMEOUT (-6) once, and the same context must step on normally
after the state is uploaded again -- bit for bit as a fresh context."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu

NX, NY, NZ, XL, ZL, RE, DT = 48, 65, 48, 4 * np.pi, 2 * np.pi, 4200.0, 0.01
SGPU_E_TIMEOUT = -6


def test_chebyshev_gemm_wait_runs_out_and_recovers():
    from simson_b200.bla import MIXED, Channel, SimsonError
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, 0.05, 9)
    ch = Channel(NX, NY, NZ, RE, XL, ZL, DT, precision=MIXED)
    fresh = Channel(NX, NY, NZ, RE, XL, ZL, DT, precision=MIXED)
    try:
        ch.set_velocity(u, v, w)
        ch.start()
        ch.set_wait_limit(1000, test_timeout=True)
        ch.substep()  # step 3's Chebyshev GEMMs run out
        with pytest.raises(SimsonError) as e:
            ch.scalars()
        assert e.value.code == SGPU_E_TIMEOUT
        # reported once: a second read sees only what the invalid substep left
        # (here a non-finite pressure gradient), not the timeout again
        try:
            ch.scalars()
        except SimsonError as again:
            assert again.code != SGPU_E_TIMEOUT
        # normal limits, state restored: the context steps as a fresh one
        ch.set_wait_limit(0, test_timeout=False)
        for c in (ch, fresh):
            c.set_velocity(u, v, w)
            c.start()
            c.step(2)
            c.scalars()
        for a, b in zip(ch.state(5), fresh.state(5)):
            assert np.array_equal(a, b)
    finally:
        ch.close()
        fresh.close()


def test_learned_model_wait_runs_out_and_recovers():
    from sgs_mlp import init_weights, mlp_forward
    from simson_b200.bla import Channel, SimsonError
    w = init_weights(3)
    x = np.random.default_rng(5).standard_normal((1000, 10)).astype(np.float32)
    ch = Channel(16, 17, 16, 4200.0, 2 * np.pi, np.pi, 0.005)
    try:
        ch.set_wait_limit(1000, test_timeout=True)
        with pytest.raises(SimsonError) as e:
            ch.sgs_mlp_eval(w, x)
        assert e.value.code == SGPU_E_TIMEOUT
        ch.set_wait_limit(0, test_timeout=False)
        y = ch.sgs_mlp_eval(w, x)
        want = mlp_forward(x, w)
        assert np.linalg.norm(y - want) <= 1e-3 * np.linalg.norm(want)
    finally:
        ch.close()


def test_learned_model_in_the_step_reports_the_timeout():
    from sgs_mlp import init_weights
    from simson_b200.bla import Channel, SimsonError
    u, v, w = channel_field(32, 33, 32, 2 * np.pi, np.pi, 0.1, 12, kmax=14)
    ch = Channel(32, 33, 32, 4200.0, 2 * np.pi, np.pi, 0.005)
    try:
        ch.set_velocity(u, v, w)
        ch.start()
        ch.set_sgs_mlp(init_weights(7, scale=1e-3), s_in=0.5, s_y=2.0)
        ch.set_wait_limit(1000, test_timeout=True)
        ch.substep()
        with pytest.raises(SimsonError) as e:
            ch.scalars()
        assert e.value.code == SGPU_E_TIMEOUT
        ch.set_wait_limit(0, test_timeout=False)
        ch.set_velocity(u, v, w)
        ch.start()
        ch.substep()
        ch.scalars()
    finally:
        ch.close()
