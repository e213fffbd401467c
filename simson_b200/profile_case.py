"""Run a few substeps of the channel step on one grid (for profiler captures).

    python -m simson_b200.profile_case --grid 192x129x160 --substeps 3 [--precision mixed]

Prints the per-kernel milliseconds of the last substep (CUDA events).
"""
import argparse

import numpy as np

from .bla import FP64, MIXED, Channel
from .fields import channel_field


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="192x129x160")
    ap.add_argument("--substeps", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    a = ap.parse_args()
    nx, ny, nz = (int(v) for v in a.grid.split("x"))
    xl, zl = 4 * np.pi, 2 * np.pi
    ch = Channel(nx, ny, nz, 4200.0, xl, zl, 0.005, precision=MIXED if a.precision == "mixed" else FP64)
    ch.set_velocity(*channel_field(nx, ny, nz, xl, zl, 0.1, 2))
    ch.prhs()
    ch.substeps(a.substeps)
    ch.profile(True)
    ch.substeps(1)
    print({k: round(v[0], 4) for k, v in ch.profile_read().items() if v[1]})
    ch.close()


if __name__ == "__main__":
    main()
