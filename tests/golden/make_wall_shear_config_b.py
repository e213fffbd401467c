"""Generates tests/golden/wall_shear_config_b.npz: the reference's own
statistics over 2000 RK3 steps of the Re_tau ~ 180 channel (192x129x160,
box 4pi x 2 x 2pi, Re_cl 4200, constant flux, dt 0.005, seeded perturbation
of rms 0.1, seed 2), run by the translated reference (oracle/_ref) on the
host cores of the machine that has the reference sources.

Every 20 steps (the state after 19, 39, ..., 1999 steps) it keeps the
amp.stat row of bla/wampbl.f:276-278 (oracle/amp_row.py on the reference's
amp(nyp,20) from bla/boxamp.f, sampled inside the first substep of a step,
bla/nonlinbl.f:429-432 with iamp = 3), and the whole amp(nyp,20) of the last
sample.  The GPU test (tests/test_gpu_wall_shear.py) takes the same samples of
its own run and compares the mean wall shear, h+ and the bulk Reynolds
number over the 2000 steps.

Run: python tests/golden/make_wall_shear_config_b.py [threads]
(about 20 minutes on 8 cores).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

NX, NY, NZ = 192, 129, 160
XL, ZL, RE, DT, RMS, SEED = 4 * np.pi, 2 * np.pi, 4200.0, 0.005, 0.1, 2
STEPS, EVERY = 2000, 20


def main():
    from amp_row import amp_row
    from refsim import RefSim
    from simson_b200.fields import channel_field
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    ref = RefSim(NX, NY, NZ, RE, XL, ZL, DT, threads=threads)
    u, v, w = channel_field(NX, NY, NZ, XL, ZL, RMS, SEED)
    ref.set_velocity(u, v, w)
    ref.start()
    ref.set_iamp(3)
    rows, steps_at = [], []
    t0 = time.time()
    last_amp = None
    for s in range(STEPS):
        ref.step(1)  # boxamp of the state after s steps runs inside this step's first substep
        if (s + 1) % EVERY == 0:
            amp = ref.amp()
            sc = ref.scalars()
            rows.append(amp_row(amp, s * DT, RE, sc["px"]))
            steps_at.append(s)
            last_amp = amp
            print(f"step {s}: tau1 {rows[-1][13]:.6e} tau2 {rows[-1][14]:.6e} h+ {rows[-1][10]:.4f} "
                  f"({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(os.path.join(HERE, "wall_shear_config_b.npz"), rows=np.array(rows),
                        steps=np.array(steps_at), last_amp=last_amp,
                        config=np.array([NX, NY, NZ, XL, ZL, RE, DT, RMS, SEED, STEPS, EVERY], dtype=np.float64))


if __name__ == "__main__":
    main()
