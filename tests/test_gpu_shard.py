"""The multi-GPU step (simson_b200/shard.py) emulated on one device: P shard
contexts, each computing step 2 on its xz-planes and step 3 on its kz planes,
with the two block exchanges of every substep done as device copies (the same
blocks sgpu_copy_block packs for NCCL in a multi-GPU run).  After two steps
the assembled state must equal a single context's bit for bit, FP64 and
mixed."""
import numpy as np
import pytest

from simson_b200.fields import channel_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_shards_equal_one_context(precision, nranks):
    from simson_b200.bla import Channel
    from simson_b200.shard import LocalShards
    nx, ny, nz = 48, 65, 48
    xl, zl = 4 * np.pi, 2 * np.pi
    u, v, w = channel_field(nx, ny, nz, xl, zl, 0.05, 5)

    def make():
        ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.01, precision=precision)
        ch.set_velocity(u, v, w)
        ch.prhs()
        return ch

    one = make()
    try:
        one.step(2)
        ref = one.state(7)
        px = one.scalars()["px"]
    finally:
        one.close()
    sh = LocalShards(make, nranks, "cuda:0")
    try:
        sh.step(2)
        got = sh.state(7)
        px_sh = sh.chs[0].scalars()["px"]  # the shard that owns kz = 0
    finally:
        sh.close()
    # every plane and every pencil is computed by one context with the same
    # kernels and the same arithmetic (the tensor-core transforms give each
    # column the same result whatever tile it sits in): bit for bit
    diffs = [float(np.abs(got[k] - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-300)) for k in range(7)]
    print(precision, nranks, "max relative difference per slot:", ["%.1e" % d for d in diffs])
    assert max(diffs) == 0.0, diffs
    assert px_sh == px
