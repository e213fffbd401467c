"""CUDA-graph replay of whole RK3 steps (sgpu_step_rk) against direct
launches: the same kernels in the same order, so the state, px and the CFL
number must agree bit for bit.  The sequence starts and ends off a step
boundary (single substeps through sgpu_nonlin / sgpu_linear) so that both
the replayed steps and the directly launched substeps around them run, and
switches the LES model on half way (the captured step must be dropped)."""
import os

import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


def run(graphs, precision):
    from simson_b200.bla import Channel
    nx, ny, nz = 48, 65, 48
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.05, 5)
    old = os.environ.get("SIMSON_GRAPHS")
    os.environ["SIMSON_GRAPHS"] = "1" if graphs else "0"
    try:
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=precision)
    finally:
        if old is None:
            del os.environ["SIMSON_GRAPHS"]
        else:
            os.environ["SIMSON_GRAPHS"] = old
    try:
        ch.set_velocity(u, v, w)
        ch.prhs()
        ch.step(3)
        ch.nonlinbl()
        ch.linearbl()
        ch.step(3)           # two direct substeps, two replayed steps, one direct substep
        ch.set_les(iles=1)
        ch.step(3)
        launches = ch.launches()
        return ch.state(7), ch.scalars(), launches
    finally:
        ch.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_runs_are_deterministic(precision):
    """Same inputs, same bytes: two runs of the same sequence (no atomics
    whose order reaches a result: the CFL maximum is order-free)."""
    s1, sc1, _ = run(True, precision)
    s2, sc2, _ = run(True, precision)
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    assert sc1 == sc2


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_equals_direct_launches(precision):
    s_g, sc_g, l_g = run(True, precision)
    s_d, sc_d, l_d = run(False, precision)
    for a, b in zip(s_g, s_d):
        assert np.array_equal(a, b)
    assert sc_g["px"] == sc_d["px"] and sc_g["cfl"] == sc_d["cfl"]
    assert l_g == l_d
