"""A-posteriori test of the learned SGS model (no reference counterpart):
LES of the Re_tau ~ 395 channel at 64x97x64 (box 2pi x 2 x pi, Re_cl 9000,
dt 0.005, 5000 steps = 25 time units) from the seeded field of the DNS
workload, with
  * the learned model (trained on the GPU on box-filtered fields of the
    library's own FP64 DNS at 384x193x384, tests/golden/make_learned_sgs.py)
    and its per-plane fallback to dynamic Smagorinsky,
  * the plain model, dynamic Smagorinsky of bla/les.f,
  * no model,
against the filtered DNS (the DNS truncated to the LES's modes, at the LES's
Gauss-Lobatto points), mean U and rms u', v', w' profiles averaged over the
second half of the run (t = 12.5 .. 25, the turbulent phase after the
transition at t ~ 4-10).

Gates: the learned model's mean profile within 3 % of the filtered DNS (max
over y, relative to the centreline velocity); its rms profiles closer to the
filtered DNS than the plain model's and the no-model run's (relative L2 over
y, the three components together), and within 12 % (max over y relative to
the profile's peak).  The measured deviations are printed."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "learned_sgs_re395.npz")
sys.path.insert(0, os.path.join(HERE, "golden"))


def deviations(prof, dns):
    n = min(len(prof), len(dns))
    half = n // 2
    les, ref = prof[half:n].mean(axis=0), dns[half:n].mean(axis=0)
    dmax = [float(np.abs(les[k] - ref[k]).max() / np.abs(ref[k]).max()) for k in range(4)]
    rms_l2 = float(np.linalg.norm(les[1:] - ref[1:]) / np.linalg.norm(ref[1:]))
    return dmax, rms_l2


@pytest.mark.slow
def test_learned_les_against_filtered_dns_and_plain_model():
    from make_learned_sgs import DNS, LES_DT, run_les
    from sgs_mlp import mlp_unpack
    g = np.load(GOLDEN)
    weights = {k: v.astype(np.float32) for k, v in mlp_unpack(g["params"]).items()}
    scales = (float(g["s_in"]), float(g["s_y"]), float(g["s_out"]))
    dns_steps, sample_every = int(g["config"][0]), int(g["config"][1])
    steps = int(round(dns_steps * DNS["dt"] / LES_DT))
    every = int(round(sample_every * DNS["dt"] / LES_DT))
    dns = g["dns_prof"]
    out = {}
    for model in ("mlp_fb", "dyn", "none"):
        prof, info = run_les(model, weights, scales, steps, every)
        assert prof is not None, (model, info)
        out[model] = deviations(prof, dns)
        print(model, "max deviation U, urms, vrms, wrms:", ["%.3f" % d for d in out[model][0]],
              "rms L2 %.3f" % out[model][1], "switched planes per sample:" if info else "", info or "")
    (dmax, l2) = out["mlp_fb"]
    assert dmax[0] <= 0.03, dmax
    assert max(dmax[1:]) <= 0.12, dmax
    assert l2 < out["dyn"][1] and l2 < out["none"][1], out
