"""Generates tests/golden/learned_sgs_re395.npz on a GPU: the learned SGS
model trained on box-filtered fields of the library's own FP64 DNS of the
Re_tau ~ 395 channel, and the filtered-DNS profiles that the LES at
64x97x64 is judged against.

1. DNS: 384x193x384, box 2pi x 2 x pi, Re_cl 9000, constant flux,
   dt 0.002, the seeded perturbation of rms 0.1 (seed 3, the bench field),
   DNS_STEPS steps of the library's step (precision DNS_PRECISION).
   Every SAMPLE_EVERY steps it keeps
   * the filtered-DNS profiles: the state truncated to the modes the LES grid
     holds (kx < 32, |kz| < 32), at the LES's 97 Gauss-Lobatto points (every
     other point of the 193: the 97-point grid is a subset), mean U(y) and
     rms u', v', w' (Parseval over the kept modes);
   * from TRAIN_FROM on, a training snapshot: sgpu_box_filter_sample with
     f = 6 (6 x 6 DNS points = one LES cell in x and z): the nine filtered
     velocity gradients and the wall distance in, the box-filter stress
     <u_i u_j> - <u_i><u_j> out.
2. Training on the GPU (sgpu_sgs_mlp_train, the project's own forward,
   backward and Adam kernels): a random subset of TRAIN_SAMPLES snapshot
   points, the deviatoric stress as target (the trace only adds a gradient
   to H, which the velocity-vorticity equations do not see), features
   scaled by 1/std of the gradients, targets by their std.
3. The LES at 64x97x64 (same box and Re, dt LES_DT) from the same seeded
   field (the generator draws the same continuous field on any grid) with
   each model, for the report printed at the end; tests/test_gpu_learned_les.py
   runs the same comparison against this file.

Run: python tests/golden/make_learned_sgs.py  (about 10 minutes on one B200;
DNS_STEPS, SAMPLE_EVERY, TRAIN_FROM, TRAIN_SAMPLES, TRAIN_ITERS, DNS_PRECISION
and LEARNED_SGS_OUT override the defaults).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

OUT = os.environ.get("LEARNED_SGS_OUT", os.path.join(HERE, "learned_sgs_re395.npz"))
DNS = dict(nx=384, ny=193, nz=384, re=9000.0, xl=2 * np.pi, zl=np.pi, dt=0.002, rms=0.1, seed=3)
LES = dict(nx=64, ny=97, nz=64)
LES_DT = 0.005
DNS_STEPS = int(os.environ.get("DNS_STEPS", 12500))
SAMPLE_EVERY = int(os.environ.get("SAMPLE_EVERY", 500))
TRAIN_FROM = int(os.environ.get("TRAIN_FROM", 6000))
TRAIN_SAMPLES = int(os.environ.get("TRAIN_SAMPLES", 2_000_000))
TRAIN_ITERS = int(os.environ.get("TRAIN_ITERS", 3000))
DNS_PRECISION = os.environ.get("DNS_PRECISION", "fp64")
BOX = 6


def filtered_profiles(state, nx_keep, nz_keep, ystride):
    """Mean U(y) and rms of u', v', w' of the modes kx < nx_keep/2,
    |kz| < nz_keep/2 of a (nz, ny, nx/2) state, at every ystride-th point."""
    u = state[0]
    nz = u.shape[0]
    kz = np.r_[0:nz_keep // 2, nz - nz_keep // 2 + 1:nz]
    out = [u[0, ::ystride, 0].real.copy()]
    for f in state[:3]:
        a = f[kz][:, ::ystride, :nx_keep // 2]
        p = np.abs(a) ** 2
        p[:, :, 1:] *= 2.0
        p[0, :, 0] = 0.0
        out.append(np.sqrt(p.sum(axis=(0, 2))))
    return np.stack(out)  # (4, ny_les): U, urms, vrms, wrms


def run_les(model, weights, scales, steps, every, precision="fp64", bound=0.0):
    from simson_b200.bla import FP64, MIXED, Channel
    from simson_b200.fields import channel_field
    nx, ny, nz = LES["nx"], LES["ny"], LES["nz"]
    u, v, w = channel_field(nx, ny, nz, DNS["xl"], DNS["zl"], DNS["rms"], DNS["seed"])
    ch = Channel(nx, ny, nz, DNS["re"], DNS["xl"], DNS["zl"], LES_DT, precision=FP64 if precision == "fp64" else MIXED)
    prof, switched = [], []
    try:
        ch.set_velocity(u, v, w)
        ch.start()
        if model == "dyn":
            ch.set_les(iles=2, cs=0.0, ineg=1)
        elif model in ("mlp", "mlp_fb"):
            ch.set_sgs_mlp(weights, s_in=scales[0], s_y=scales[1], s_out=scales[2])
            if model == "mlp_fb":
                ch.set_sgs_fallback(bound=bound, cs=0.0, ineg=1)
        done = 0
        while done < steps:
            ch.step(every)
            done += every
            sc = ch.scalars()
            if not np.isfinite(sc["px"]):
                return None, done
            prof.append(filtered_profiles(ch.state(3), nx, nz, 1))
            if model == "mlp_fb":
                switched.append(int(ch.sgs_fallback_planes()[0].sum()))
    except RuntimeError as e:
        print(model, "stopped:", e)
        return None, done
    finally:
        ch.close()
    return np.array(prof), switched


def main():
    from sgs_mlp import init_weights, mlp_pack, mlp_unpack
    from simson_b200.bla import FP64, MIXED, Channel
    from simson_b200.fields import channel_field
    t_start = time.time()
    d = DNS
    ch = Channel(d["nx"], d["ny"], d["nz"], d["re"], d["xl"], d["zl"], d["dt"],
                 precision=MIXED if DNS_PRECISION == "mixed" else FP64)
    u, v, w = channel_field(d["nx"], d["ny"], d["nz"], d["xl"], d["zl"], d["rms"], d["seed"])
    ch.set_velocity(u, v, w)
    ch.start()
    dns_prof, dns_t, hplus, feats, targs = [], [], [], [], []
    rng = np.random.default_rng(0)
    done = 0
    while done < DNS_STEPS:
        ch.step(SAMPLE_EVERY)
        done += SAMPLE_EVERY
        sc = ch.scalars()
        _, row = ch.amplitudes()
        hplus.append(row["hplus"])
        dns_prof.append(filtered_profiles(ch.state(3), LES["nx"], LES["nz"], 2))
        dns_t.append(done * d["dt"])
        if done >= TRAIN_FROM:
            f, t = ch.box_filter_sample(BOX)
            f, t = f.reshape(-1, 10), t.reshape(-1, 6)
            keep = rng.random(f.shape[0]) < 0.25
            feats.append(f[keep])
            targs.append(t[keep])
        print(f"DNS step {done}: t {done * d['dt']:.2f} h+ {row['hplus']:.1f} cfl {sc['cfl']:.3f} "
              f"urms(center) {dns_prof[-1][1][48]:.4f} ({time.time() - t_start:.0f} s)", flush=True)
    # training set: deviatoric stress, scaled
    x = np.concatenate(feats).astype(np.float64)
    tau = np.concatenate(targs).astype(np.float64)
    if x.shape[0] > TRAIN_SAMPLES:
        pick = rng.choice(x.shape[0], TRAIN_SAMPLES, replace=False)
        x, tau = x[pick], tau[pick]
    tr = (tau[:, 0] + tau[:, 3] + tau[:, 5]) / 3.0
    dev = tau - tr[:, None] * np.array([1, 0, 0, 1, 0, 1.0])
    s_in = float(1.0 / x[:, :9].std())
    s_y = 1.0
    s_out = float(dev.std())
    xs = np.concatenate([x[:, :9] * s_in, x[:, 9:] * s_y], axis=1)
    ys = dev / s_out
    p0 = mlp_pack(init_weights(0, scale=0.1))
    z = np.zeros_like(p0)
    _, _, _, _, loss0, _ = ch.sgs_mlp_train(p0, z, z, 0, xs, ys, 0, 1e-3)
    p, m, vv, step, loss, _ = ch.sgs_mlp_train(p0, z, z, 0, xs, ys, TRAIN_ITERS, 1e-3)
    print(f"training: {xs.shape[0]} samples, loss {loss0:.4f} -> {loss:.4f} after {step} Adam steps "
          f"({time.time() - t_start:.0f} s)", flush=True)
    ch.close()
    weights = {k: v.astype(np.float32) for k, v in mlp_unpack(p).items()}
    scales = (s_in, s_y, s_out)
    dns_prof = np.array(dns_prof)
    les_steps = int(round(DNS_STEPS * d["dt"] / LES_DT))
    les_every = int(round(SAMPLE_EVERY * d["dt"] / LES_DT))
    report = {}
    for model in ("none", "dyn", "mlp", "mlp_fb"):
        prof, info = run_les(model, weights, scales, les_steps, les_every)
        if prof is None:
            print(f"LES {model}: diverged by step {info}")
            report[model] = None
            continue
        n = min(len(prof), len(dns_prof))
        half = n // 2
        les_mean, dns_mean = prof[half:n].mean(axis=0), dns_prof[half:n].mean(axis=0)
        err = [float(np.abs(les_mean[k] - dns_mean[k]).max() / np.abs(dns_mean[k]).max()) for k in range(4)]
        report[model] = err
        print(f"LES {model}: max deviation from filtered DNS over the second half (U, urms, vrms, wrms): "
              + " ".join(f"{e:.3f}" for e in err) + (f" switched planes {info}" if info else ""), flush=True)
    np.savez_compressed(OUT, params=p, s_in=s_in, s_y=s_y, s_out=s_out, dns_prof=dns_prof, dns_t=np.array(dns_t),
                        hplus=np.array(hplus), loss=np.array([loss0, loss]), train_samples=xs.shape[0],
                        config=np.array([DNS_STEPS, SAMPLE_EVERY, TRAIN_FROM, BOX, LES_DT], dtype=np.float64))
    print(f"wrote {OUT} ({time.time() - t_start:.0f} s)")


if __name__ == "__main__":
    main()
