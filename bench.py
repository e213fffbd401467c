#!/usr/bin/env python
"""Benchmark of the channel time step: RK3 steps/s at 384x193x384.

Workload (the production-DNS configuration the headline metric is quoted on):
temporal channel, 384x193x384 modes (3/2-rule grid 576x193x576), box
2pi x 2 x pi, Re_cl = 9000, constant flow rate, dt = 0.002, seeded
divergence-free perturbation of rms 0.1 on laminar Poiseuille flow.  One
"step" is one full RK3 step (three substeps of nonlinear step 2 + implicit
step 3).  The state (1.6 GB in FP64) is far larger than L2, so no flush is
needed between steps.

Arms:
  own (default)   the CUDA step through the C ABI, state resident in HBM;
                  ``e2e`` repeats it through the same ABI with the whole state
                  uploaded from pinned host memory and downloaded every step
                  (sgpu_offload_steps: the copies of consecutive steps overlap
                  per slot, PCIe being full duplex).
  --impl reference  the reference's own CPU implementation of the step (the
                  translated Fortran, oracle/_ref) on all host cores, OpenMP.

Multi-GPU: by default the step runs as independent replicas, one per rank
(weak scaling); --shard splits one channel over the ranks (z-slab shards with
two NCCL block all-to-alls per substep, simson_b200/shard.py; strong scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

REF_MAX_STEPS = 20
WORKLOAD = dict(nx=384, ny=193, nz=384, re=9000.0, xl=2 * np.pi, zl=np.pi, dt=0.002, rms=0.1, seed=3)
METRIC = "RK3 steps/s at 384x193x384"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def substep_bytes(nc, precision):
    """Algorithmic main-storage traffic of one substep: step 2 reads 5 fields
    and writes 3, step 3 reads 5 and writes 7 (20 field passes), at the
    storage precision of each field: FP64 everywhere, or under the mixed
    path FP32 for u, v, w, omega_x, omega_z and H (16 passes) and FP64 for
    p_v, p_omega (4 passes)."""
    if precision == "fp64":
        return 20 * nc * 16
    return 16 * nc * 8 + 4 * nc * 16


def kernel_bytes(name, w, precision="fp64"):
    """Algorithmic (compulsory) HBM bytes of one launch of each kernel."""
    nx2, ny, nz = w["nx"] // 2, w["ny"], w["nz"]
    nzp = nz + nz // 2
    c = 16 if precision == "fp64" else 8
    fld = nx2 * ny * nz * c          # one spectral field
    fine = nx2 * ny * nzp * c        # one z-transformed field on the 3/2 z grid
    f64 = nx2 * ny * nz * 16         # a field kept in FP64 (Chebyshev-space scratch of step 3)
    # Chebyshev-space fields of step 3: FP64, or FP32 for H and for the
    # u, v, w, omega outputs under the mixed path
    cf = f64 if precision == "fp64" else fld
    return {
        "zinv": 5 * fld + 6 * fine,
        "xpass": 6 * fine + 3 * fine,
        "zfwd": 3 * fine + 3 * fld,
        "cheb_fwd": 3 * fld + 3 * cf,
        # H1-H3 and p_v, p_omega in; u, v, w, omega_x, omega_z and p_v, p_omega out
        "pencil": 3 * cf + 2 * f64 + 5 * cf + 2 * f64,
        "cheb_inv": 5 * cf + 5 * fld,
    }.get(name)


def own_arm(args, rank, world, precision):
    from simson_b200.bla import Channel, PinnedArray, FP64, MIXED
    from simson_b200.fields import channel_field

    w = WORKLOAD
    prec = MIXED if precision == "mixed" else FP64
    dev = int(os.environ.get("LOCAL_RANK", 0))
    ch = Channel(w["nx"], w["ny"], w["nz"], w["re"], w["xl"], w["zl"], w["dt"], precision=prec, device=dev)
    u, v, wv = channel_field(w["nx"], w["ny"], w["nz"], w["xl"], w["zl"], w["rms"], w["seed"] + rank)
    ch.set_velocity(u, v, wv)
    ch.prhs()
    for _ in range(args.warmup):
        ch.step(1)
    ch.sync()
    dist_barrier(world)
    clk = ClockSampler(dev)
    clk.start()
    l0 = ch.launches()
    ch.record(0)
    ch.step(args.steps)
    ch.record(1)
    ms = ch.elapsed_ms(0, 1)
    launches = ch.launches() - l0
    clocks = clk.stop()
    ms = dist_max(ms, world)
    sc = ch.scalars()
    uvw = ch.state(3)  # after warm-up + timed steps, for the mixed-vs-FP64 comparison
    # per-kernel times (a separate, profiled run of 2 steps)
    ch.profile(True)
    ch.step(2)
    prof = ch.profile_read()
    ch.profile(False)
    # one xy-statistics sample (boxxys on every plane), outside the timed
    # steps: the first call sets up its buffers
    ch.xys_sample()
    ch.sync()
    ch.record(0)
    for _ in range(3):
        ch.xys_sample()
    ch.record(1)
    xys_ms = ch.elapsed_ms(0, 1) / 3
    # one pressure computation (nonlinp + linearp) including its download
    # into page-locked host buffers
    pshape = (w["nz"], w["ny"], w["nx"] // 2)
    p_re, p_im = PinnedArray(pshape), PinnedArray(pshape)
    ch.pressure_raw(p_re.ptr, p_im.ptr)
    ch.record(0)
    ch.pressure_raw(p_re.ptr, p_im.ptr)
    ch.record(1)
    press_ms = ch.elapsed_ms(0, 1)
    p_re.free()
    p_im.free()
    # end-to-end through the public API with host buffers
    nslots = 7
    shape = (nslots, w["nz"], w["ny"], w["nx"] // 2)
    hr = PinnedArray(shape)
    hi = PinnedArray(shape)
    ch.download_raw(hr.ptr, hi.ptr, nslots)
    e2e_steps = max(2, min(args.steps, 10))
    ch.sync()
    # every step uploads the 7 slots from the pinned host arrays and downloads
    # the result into them (sgpu_offload_steps; the copies of consecutive
    # steps overlap per slot)
    ch.offload_steps(hr.ptr, hi.ptr, 1)  # warm-up: streams and events
    t0 = time.perf_counter()
    ch.offload_steps(hr.ptr, hi.ptr, e2e_steps)
    e2e_s = time.perf_counter() - t0
    e2e_s = dist_max(e2e_s * 1000.0, world) / 1000.0
    nbytes = int(np.prod(shape)) * 8 * 2
    hr.free()
    hi.free()
    finite = bool(np.isfinite(sc["px"]))
    ch.close()
    return dict(ms=ms, launches=launches, clocks=clocks, prof=prof, e2e_s=e2e_s, e2e_steps=e2e_steps,
                e2e_bytes=nbytes, scalars=sc, finite=finite, uvw=uvw, xys_ms=xys_ms,
                press_ms=press_ms)


LES_WORKLOAD = dict(nx=64, ny=97, nz=64, re=9000.0, xl=2 * np.pi, zl=np.pi, dt=0.005, rms=0.1, seed=3)
LEARNED_WEIGHTS = os.path.join(ROOT, "tests", "golden", "learned_sgs_re395.npz")


def learned_model():
    """The learned SGS network trained on the DNS of the Re_tau ~ 395 channel
    (tests/golden/make_learned_sgs.py): (weights, (s_in, s_y, s_out), label);
    without that file, the eddy-viscosity weight set of oracle/sgs_mlp.py
    (the same network size and cost)."""
    if os.path.exists(LEARNED_WEIGHTS):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from sgs_mlp import mlp_unpack
        g = np.load(LEARNED_WEIGHTS)
        w = {k: v.astype(np.float32) for k, v in mlp_unpack(g["params"]).items()}
        return w, (float(g["s_in"]), float(g["s_y"]), float(g["s_out"])), "trained on the Re_tau~395 DNS"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from sgs_mlp import viscosity_weights
    return viscosity_weights(1e-5), (0.2, 1.0, 1.0), "eddy-viscosity weight set"


def setup_les(ch, model):
    if model == "adm":
        ch.set_les(iles=1)
    elif model == "dyn":
        ch.set_les(iles=2)
    elif model == "hpf":
        ch.set_les(iles=3, cs=0.1)
    elif model == "hpf_dyn":
        ch.set_les(iles=3, cs=0.0)
    elif model in ("mlp", "mlp_fb"):
        w, (s_in, s_y, s_out), _ = learned_model()
        ch.set_sgs_mlp(w, s_in=s_in, s_y=s_y, s_out=s_out)
        if model == "mlp_fb":
            ch.set_sgs_fallback(bound=0.0, cs=0.0, ineg=1)


def les_arm(steps, warmup):
    """RK3 steps/s of the LES configuration 64x97x64 (Re_cl 9000, the box of
    the 384x193x384 workload) with each SGS model: ADM-RT and dynamic
    Smagorinsky with the reference's sgs.i defaults, the HPF eddy viscosity
    (fixed cs = 0.1 and dynamic), the learned model alone and with its
    per-plane fallback to dynamic Smagorinsky."""
    from simson_b200.bla import Channel, FP64, MIXED
    from simson_b200.fields import channel_field
    w = LES_WORKLOAD
    u, v, wv = channel_field(w["nx"], w["ny"], w["nz"], w["xl"], w["zl"], w["rms"], w["seed"])
    out = {}
    variants = [("no_model_fp64", FP64, None), ("adm_rt_fp64", FP64, "adm"), ("dyn_smagorinsky_fp64", FP64, "dyn"),
                ("hpf_fixed_fp64", FP64, "hpf"), ("hpf_dynamic_fp64", FP64, "hpf_dyn"),
                ("learned_mlp_fp64", FP64, "mlp"), ("learned_mlp_fallback_fp64", FP64, "mlp_fb"),
                ("dyn_smagorinsky_mixed", MIXED, "dyn"), ("learned_mlp_mixed", MIXED, "mlp"),
                ("learned_mlp_fallback_mixed", MIXED, "mlp_fb"), ("no_model_mixed", MIXED, None)]
    for tag, prec, model in variants:
        ch = Channel(w["nx"], w["ny"], w["nz"], w["re"], w["xl"], w["zl"], w["dt"], precision=prec)
        ch.set_velocity(u, v, wv)
        if model in ("adm", "hpf", "hpf_dyn"):
            setup_les(ch, model)  # before prhs: it filters the start-up velocities
        ch.prhs()
        if model not in ("adm", "hpf", "hpf_dyn"):
            setup_les(ch, model)
        for _ in range(warmup):
            ch.step(1)
        ch.sync()
        ch.record(0)
        ch.step(steps)
        ch.record(1)
        ms = ch.elapsed_ms(0, 1)
        out[tag] = {"steps_per_s": steps / (ms / 1000.0), "ms_per_step": ms / steps}
        ch.close()
    v = out
    ratio = {k: v[k]["steps_per_s"] / v["dyn_smagorinsky_fp64"]["steps_per_s"]
             for k in ("learned_mlp_fp64", "learned_mlp_fallback_fp64", "learned_mlp_mixed",
                       "learned_mlp_fallback_mixed")}
    return {"workload": "temporal channel 64x97x64, 2pi x 2 x pi, Re_cl 9000, dt 0.005, the seeded rms 0.1 "
                        "field of the DNS workload (the learned-LES configuration)", "steps": steps,
            "warmup": warmup, "learned_weights": learned_model()[2], "variants": out,
            "learned_over_dyn_smagorinsky_fp64": ratio}


def shard_arm(args, rank, world, precision):
    """One channel of the workload split over the ranks (simson_b200.shard):
    every rank uploads the same field and runs prhs, then each substep moves
    the two block all-to-alls over NCCL around its step-2 planes and step-3
    kz planes.  Timed with CUDA events on each rank's stream, max over ranks."""
    from simson_b200.bla import Channel, FP64, MIXED
    from simson_b200.fields import channel_field
    from simson_b200.shard import ShardedChannel

    w = WORKLOAD
    dev = int(os.environ.get("LOCAL_RANK", 0))
    ch = Channel(w["nx"], w["ny"], w["nz"], w["re"], w["xl"], w["zl"], w["dt"],
                 precision=MIXED if precision == "mixed" else FP64, device=dev)
    u, v, wv = channel_field(w["nx"], w["ny"], w["nz"], w["xl"], w["zl"], w["rms"], w["seed"])
    ch.set_velocity(u, v, wv)
    ch.prhs()
    sc = ShardedChannel(ch, rank, world, f"cuda:{dev}")
    sc.step(args.warmup)
    ch.sync()
    dist_barrier(world)
    clk = ClockSampler(dev)
    clk.start()
    l0 = ch.launches()
    b0 = sc.bytes_moved
    ch.record(0)
    sc.step(args.steps)
    ch.record(1)
    ms = dist_max(ch.elapsed_ms(0, 1), world)
    clocks = clk.stop()
    out = dict(ms=ms, bytes=sc.bytes_moved - b0, launches=ch.launches() - l0, clocks=clocks)
    ch.close()
    return out


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_max(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference(steps, threads, sample_note, warmup_substeps=1):
    """Time the reference's own implementation (translated Fortran) on host
    cores: `steps` full RK3 steps after `warmup_substeps` untimed substeps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from build_ref import REF_BLA
    from refsim import RefSim
    from simson_b200.fields import channel_field
    w = WORKLOAD
    ref = RefSim(w["nx"], w["ny"], w["nz"], w["re"], w["xl"], w["zl"], w["dt"], threads=threads,
                 build=os.path.isdir(REF_BLA))
    u, v, wv = channel_field(w["nx"], w["ny"], w["nz"], w["xl"], w["zl"], w["rms"], w["seed"])
    ref.set_velocity(u, v, wv)
    ref.start()
    for _ in range(warmup_substeps):
        ref.substep()  # page faults, caches
    t0 = time.perf_counter()
    ref.step(steps)
    dt = time.perf_counter() - t0
    return dict(value=steps / dt, unit="steps/s", cores=threads, kind="reference", steps=steps,
                sample=f"{sample_note}: {steps} full RK3 steps ({3 * steps} substeps) after {warmup_substeps} "
                       f"warm-up substep(s), translated reference bla (gcc -O3 -fopenmp, the reference's own "
                       f"Fortran translated to C: no Fortran compiler exists on either machine, so bla's own "
                       f"'Wall time' lines cannot be used), {threads} threads")


def profile_case(grid, substeps, precision, les=None):
    """A few substeps of the channel step on one grid, for profiler captures
    (ncu -k ... -s ... python bench.py --case GRID): prints the per-kernel
    milliseconds of the last substep (CUDA events).  les: an SGS model
    (adm, dyn, mlp, mlp_fb) on the box and Re of the LES configuration."""
    from simson_b200.bla import FP64, MIXED, Channel
    from simson_b200.fields import channel_field
    nx, ny, nz = (int(v) for v in grid.split("x"))
    xl, zl, re = (4 * np.pi, 2 * np.pi, 4200.0) if not les else (2 * np.pi, np.pi, 9000.0)
    ch = Channel(nx, ny, nz, re, xl, zl, 0.005, precision=MIXED if precision == "mixed" else FP64)
    ch.set_velocity(*channel_field(nx, ny, nz, xl, zl, 0.1, 2))
    if les == "adm":
        setup_les(ch, les)
    ch.prhs()
    if les and les != "adm":
        setup_les(ch, les)
    ch.substeps(substeps)
    ch.profile(True)
    ch.substeps(1)
    print({k: round(v[0], 4) for k, v in ch.profile_read().items() if v[1]})
    ch.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                    help="both: time FP64 and mixed; value is the mixed-precision step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-les", action="store_true", help="skip the LES-configuration timings")
    ap.add_argument("--case", default=None, metavar="NXxNYxNZ",
                    help="profiling case: run --substeps substeps on this grid and print per-kernel times "
                         "(no JSON line; for ncu captures)")
    ap.add_argument("--substeps", type=int, default=3)
    ap.add_argument("--les", default=None, choices=["adm", "dyn", "mlp", "mlp_fb"],
                    help="profiling case: SGS model")
    ap.add_argument("--shard", action="store_true",
                    help="one channel split over the ranks (z-slab shards, NCCL all-to-alls; strong scaling) "
                         "instead of one replica per rank")
    args = ap.parse_args()
    if args.case:
        profile_case(args.case, args.substeps, "mixed" if args.precision == "mixed" else "fp64", args.les)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    threads = os.cpu_count() or 1
    w = WORKLOAD
    config = {"workload": "temporal channel 384x193x384 (576x193x576 dealiased), box 2pi x 2 x pi, Re_cl 9000, "
                          "cflux, dt 0.002, seeded rms 0.1 perturbation", "nx": w["nx"], "ny": w["ny"], "nz": w["nz"],
              "l2": "state 1.6 GB > L2, no flush needed",
              "parallelism": f"independent replicas x{args.gpus} (one whole channel per GPU, no exchange)"}
    if args.impl == "reference":
        if rank != 0:
            return
        # each timed step is one full RK3 step of the workload on all host
        # cores (about 1.7 s on 16 cores); at most REF_MAX_STEPS of them so
        # that the arm ends within a few minutes
        nsteps = max(1, min(args.steps, REF_MAX_STEPS))
        try:
            r = cpu_reference(nsteps, threads, "per step", warmup_substeps=3 * max(1, min(args.warmup, 1)))
        except Exception as e:  # pragma: no cover
            print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build failed: {e}"}))
            return
        line = {"metric": METRIC, "value": r["value"], "unit": "steps/s", "n_gpus": args.gpus, "steps": nsteps,
                "warmup": 1, "ms_per_step": 1000.0 / r["value"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "precision": "fp64 (the reference computes in double precision)", "impl": "reference",
                "cpu_baseline": r, "e2e": {"value": r["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if args.shard:
        prec = "mixed" if args.precision in ("both", "mixed") else "fp64"
        r = shard_arm(args, rank, world, prec)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        if rank == 0:
            config["parallelism"] = f"z-slab shards x{world} (step 2 on ny/{world} planes, step 3 on nz/{world} kz planes)"
            print(json.dumps({
                "precision": prec,
                "metric": METRIC, "value": args.steps / (r["ms"] / 1000.0), "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic", "config": config,
                "exchange_bytes_per_step_per_rank": r["bytes"] / max(args.steps, 1), "clocks": r["clocks"],
                "gpu_launches": r["launches"]}))
        return
    runs = {}
    for prec in (["fp64", "mixed"] if args.precision == "both" else [args.precision]):
        runs[prec] = own_arm(args, rank, world, prec)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    head = "mixed" if "mixed" in runs else "fp64"
    res = runs[head]
    steps_per_s = args.steps / (res["ms"] / 1000.0) * args.gpus
    ms_step = res["ms"] / args.steps
    hbm, peak_kind = peaks()
    nc = (w["nx"] // 2) * w["ny"] * w["nz"]
    prof = res["prof"]
    # dominant kernel by measured time
    dom = max((k for k in prof if k not in ("other",) and prof[k][1] > 0), key=lambda k: prof[k][0])
    dom_ms = prof[dom][0] / prof[dom][1]
    dom_bytes = kernel_bytes(dom, w, head)
    # DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    # from ncu captures of these kernels at this workload, summarised in
    # profiles/: the pencil kernel captured at 384x193x384 (one pass), the x
    # pass at 384x33x384 scaled by ny (its traffic grows with the planes)
    measured_traffic = {("mixed", "pencil"): 2.65e9 + 2.51e9, ("mixed", "xpass"): (175.25e6 + 60.25e6) * 193 / 33}
    roof = {"kernel": dom, "bound": "hbm", "unit": "GB/s", "peak": hbm, "peak_kind": peak_kind,
            "traffic": measured_traffic.get((head, dom)), "launch_ms": dom_ms}
    if dom_bytes:
        ach = dom_bytes / (dom_ms / 1000.0) / 1e9
        roof.update(achieved=ach, frac=ach / hbm, algorithmic_bytes=dom_bytes)
    else:
        roof.update(achieved=None, frac=None, algorithmic_bytes=None)
    stage_bytes = substep_bytes(nc, head)
    step_ach = 3 * stage_bytes / (ms_step / 1000.0) / 1e9
    precision_note = {"mixed": "mixed: FP32 x/z FFTs, products, Chebyshev transforms and u,v,w,omega storage; "
                               "FP64 tau solves, mean flow, partial RHS",
                      "fp64": "fp64: every transform and solve in FP64"}[head]
    line = {
        "precision": precision_note,
        "metric": METRIC, "value": steps_per_s, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64", "data": "synthetic",
        "config": config,
        "grid_point_stages_per_s": w["nx"] * w["ny"] * w["nz"] * 3 * steps_per_s,
        "roofline": roof,
        "step_roofline": {"bound": "hbm", "bytes_per_substep": stage_bytes, "achieved": step_ach, "peak": hbm,
                          "frac": step_ach / hbm, "unit": "GB/s"},
        "kernel_ms_per_substep": {k: (v[0] / max(v[1], 1)) for k, v in prof.items() if v[1]},
        "e2e": {"value": res["e2e_steps"] / res["e2e_s"] * args.gpus, "unit": "steps/s",
                "h2d_bytes_per_step": res["e2e_bytes"], "d2h_bytes_per_step": res["e2e_bytes"]},
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
        "finite": res["finite"],
        "xys_sample_ms": res["xys_ms"],
        "pressure_ms": res["press_ms"],
    }
    if "fp64" in runs and "mixed" in runs:
        r64 = runs["fp64"]
        sps64 = args.steps / (r64["ms"] / 1000.0) * args.gpus
        keep = np.ones(w["nz"], bool)
        keep[w["nz"] // 2] = False  # the oddball kz plane carries the last H in both paths; never read
        errs = [float(np.linalg.norm(runs["mixed"]["uvw"][k][keep] - r64["uvw"][k][keep]) /
                      np.linalg.norm(r64["uvw"][k][keep])) for k in range(3)]
        line["fp64"] = {"value": sps64, "ms_per_step": r64["ms"] / args.steps,
                        "kernel_ms_per_substep": {k: (v[0] / max(v[1], 1)) for k, v in r64["prof"].items() if v[1]},
                        "e2e": r64["e2e_steps"] / r64["e2e_s"] * args.gpus}
        line["mixed_over_fp64"] = steps_per_s / sps64
        line["mixed_vs_fp64_rel_l2_uvw"] = {"after_steps": args.warmup + args.steps, "u": errs[0], "v": errs[1],
                                            "w": errs[2]}
        line["gpu_launches"] += r64["launches"]
    if world == 1 and not args.no_les:
        line["les"] = les_arm(max(args.steps, 20), max(args.warmup, 3))
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_reference(3, threads, "bounded sample")
        except Exception as e:  # pragma: no cover
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
