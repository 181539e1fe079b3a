#!/usr/bin/env python
"""Benchmark: particle-steps/s of the SPH step on the 128^3 Oldroyd-B Couette workload.

Workload (the reference's headline configuration, 3D Couette flow): 128^3 lattice between
y-walls (128 x 134 x 128 = 2,195,456 particles including the wall layers), L = 1,
overlap = 3, V_wall = -0.5 / +0.5, rho = 1, c = 10, P0 = 0, eta = 0.1, zeta = 0,
np = 100, kT = 0.01, tau = 1, dt = 2e-5; synthetic initial state: the lattice with c = I
and every fluid velocity component drawn uniform in +-1e-3 c = +-0.01 from seed 2, given to
both the engine and the reference as new_sim = 1 with an input_particles.in restart file
(the only way the reference takes an initial velocity field).  A step is the reference
driver's step (main.cu:358-467): half-kick and drift, neighbour search, density, velocity
gradient, forces, dc/dt, wall forces, half-kick.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
  python bench.py --impl reference ...    # the reference's own CUDA build, same workload

value : K * N_particles * n_ranks / (max over ranks of the device time of K steps),
        measured with CUDA events on the engine's stream around one sph_step(K) call
        (CUDA-graph replay), inputs resident in HBM.  The state (~0.7 GB) is larger than
        the 126 MB L2, so no L2 flush is needed between steps.
e2e   : the same metric through the reference-facing C ABI with host buffers: every step
        calls V_Verlet_step1, neighbours_search, calculate_forces(m) with the magnetic
        moment copied from host memory, V_Verlet_step2, then reads the wall forces and the
        kinetic energy back to the host (wall-clock time).
With N > 1 GPUs every rank advances its own replica of the box (the single box does not
shard; replicas only): weak scaling, no collective in the data path.

  python bench.py --workload ensemble512 [--gpus N] [--precision fp64|mixed]

The batched workload: 512 independent 2D wall-bounded boxes (side 32..128, seeded
parameters and colloids, sph_ensemble.py) in one context per GPU, sharded over ranks by
particle-steps (strong scaling, no exchange); the JSON line adds the same boxes run one
at a time (`looped_single_box`, a sample of every 16th box) and the ratio.

  python bench.py --workload sweep [--sweep-train 20480] [--sweep-steps 2000]

Sweep points per hour: 20,480 sweep points solved by the batched solver train the
surrogate (5 heads); 65,536 query points are predicted and those on which the heads
disagree by more than 2% are re-solved; 512 held-out points re-solved by the solver give
the wall-stress error; one-at-a-time plain runs (a sample of 8) give the baseline rate.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "sph-magnetic-particles-oldroyd-b-in-cuda_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

import sph_input  # noqa: E402

WORKLOAD = dict(N=(128, 128, 128), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1,
                Vwall_bottom=-0.5, Vwall_top=0.5, rho=1.0, c=10.0, P0=0.0, eta=0.1, zeta=0.0,
                np=100.0, kT=0.01, tau=1.0, dt=2e-5)
WORKLOAD_NAME = ("couette3d_128: 128^3 Oldroyd-B Couette flow between y-walls, 2,195,456 "
                 "particles, fluid velocities seeded uniform in +-1e-3 c")
# seeded initial fluid velocities: uniform in [-VMAX, VMAX] per component, VMAX = 1e-3 c
SEED, VMAX = 2, 1e-3 * 10.0
METRIC = "particle-steps/s (128^3 Oldroyd-B Couette)"
UNIT = "particle-steps/s"
# Algorithmic bytes per particle-step of the whole step (four grid-wide phases, each
# per-particle field read once and written once): (10 d + 5 n_c + 4) P + 28 with d = 3,
# n_c = 6 conformation components, P = bytes per real.
B_ALG_STEP = {"fp64": (10 * 3 + 5 * 6 + 4) * 8 + 28, "mixed": 380}
# Algorithmic bytes per particle of one launch of the fused pair kernel (k_pairs):
# reads x, v (6 reals), Pi/d^2 (6), 1/d, p, c (6), mass (1) and the type word; writes
# f (3) and dc/dt (6).
B_ALG_PAIRS = {"fp64": (6 + 6 + 1 + 1 + 6 + 1 + 3 + 6) * 8 + 4,
               "mixed": (6 + 6 + 1) * 4 + (1 + 6 + 1 + 3 + 6) * 8 + 4}
# FP64 floating-point operations per particle of one launch of the FP64 pair kernel, counted
# by ncu on the 96^3 case of this workload (same lattice, same neighbours per particle):
# DADD + DMUL + 2 DFMA thread instructions (each per-cycle rate times the SM sub-partition's
# elapsed cycles) / particles (profiles/k_pairs_couette96_fp64.md).
FP64_PAIR_FLOP = 11626.9
# FP64 peak of the B200: 148 SMs x 64 FP64 FMA lanes (ncu's dfma peak_sustained, 9,472 per
# cycle) x 2 FLOP x the SM clock.
FP64_LANES = 9472


def clock_mhz():
    """Maximum SM clock of this pool's B200s (MEASURED_PEAKS.json), else the nominal 1965 MHz."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f).get("sm_max_mhz", 1965.0))
    return 1965.0


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
         "utilization.gpu")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, busy, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [t.strip() for t in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    clk, top = float(p[1]), float(p[2])
                except ValueError:
                    continue
                sm.append(clk)
                smax.append(top)
                try:
                    util = float(p[9]) if len(p) > 9 else 100.0
                except ValueError:
                    util = 100.0
                if util > 0:
                    busy.append(clk)
                for k, name in enumerate(names):
                    if p[5 + k].lower() == "active":
                        reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        # the median over the samples in which the GPU was busy (a sampled process that also
        # reads its input spends part of its time with the GPU idle, at idle clocks)
        return {"sm_mhz": statistics.median(busy or sm), "sm_max_mhz": max(smax),
                "samples": len(sm), "busy_samples": len(busy), "reasons": sorted(reasons)}


def write_workload(d, lattice=128):
    """The Couette input (`input`, new_sim = 1) and its seeded start (`input_particles.in`)
    in directory d; lattice < 128 gives a smaller box of the same physics, used only for ncu
    captures that must stay small.  Returns the input path; the engine, the oracle and the
    reference all read the same two files."""
    import sph_b200

    spec = dict(WORKLOAD)
    spec["N"] = (lattice, lattice, lattice)
    path, _, _ = sph_b200.write_seeded_start(d, spec, seed=SEED, vmax=VMAX)
    return path


def particles_file(input_path):
    """The restart file beside an input, or None when the input starts from the lattice."""
    p = os.path.join(os.path.dirname(input_path), "input_particles.in")
    return p if os.path.exists(p) else None


SUSPENSION_NAME = ("suspension3d_96: 96^3 Oldroyd-B fluid between walls at rest with 32 rotating "
                   "magnetic colloids of radius 4 dx (sph_input.suspension_spec, seed 11), "
                   "F0_repulsion 1e-3, F0_magnetic 5e-4")
SUSPENSION_METRIC = "particle-steps/s (96^3 magnetic suspension, 32 colloids)"
# The amplitudes as the configuration writes them (F0_repulsion 10, F0_magnetic 5) drive the
# colloids of radius 4 dx to speeds of hundreds of box lengths per unit time (the magnetic
# force is F0 / r^4 with r in box units, ~1e3 per pair at contact on a colloid of mass 3e-4)
# and one colloid leaves the box at step 154, where the reference would trap on its cell
# range check; scaled by 1e-4 the run is stable for its 2000 steps (colloid speeds below 1.2).
SUSPENSION_F0 = dict(F0_repulsion=1e-3, F0_magnetic=5e-4)


def write_suspension(d, lattice=96):
    """The 3D magnetic suspension input in directory d (lattice start, no restart file)."""
    path = os.path.join(d, "input")
    sph_input.write_input(path, **sph_input.suspension_spec(N=lattice, **SUSPENSION_F0))
    return path


class Workload:
    """A single-box benchmark workload: its name, metric and input writer."""

    def __init__(self, key, name, metric, write, lattice):
        self.key, self.name, self.metric, self.write, self.lattice = key, name, metric, write, lattice


WORKLOADS = {
    "couette3d": Workload("couette3d", WORKLOAD_NAME, METRIC, write_workload, 128),
    "suspension96": Workload("suspension96", SUSPENSION_NAME, SUSPENSION_METRIC, write_suspension,
                             96),
}


def cpu_baseline(workdir, wl, steps=1):
    """The FP64 OpenMP oracle on this host: initial forces, then `steps` timed steps."""
    import oracle

    cores = oracle.set_threads(os.cpu_count() or 1)
    inp = wl.write(workdir)
    o = oracle.Oracle(inp, particles_file(inp))
    o.run(0)
    t0 = time.perf_counter()
    o.run(steps)
    dt = time.perf_counter() - t0
    n = o.info()["N"]
    o.close()
    return {"value": n * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "CPU oracle (C99+OpenMP FP64 restatement) on the full %s workload: "
                      "initial forces untimed, then %d timed step(s), %.1f s" % (wl.key, steps, dt)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        return world, rank, local, dist
    return 1, 0, local, None


def max_over_ranks(dist, value, local):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cuda:%d" % local)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, world, rank, dist, wl):
    """The reference's own CUDA build (oracle/_ref/ref_sph: its unmodified sources driven by
    oracle/ref_harness.cu), timed with CUDA events around the step loop."""
    if rank != 0:
        return 0
    # FP64: the reference as shipped; with --precision mixed, its FP32 configuration
    # (real = float in src/config.h), the same-precision baseline of the mixed engine
    fp32 = args.precision != "fp64"
    rel = os.path.join("oracle", "_ref", "fp32", "ref_sph") if fp32 else \
        os.path.join("oracle", "_ref", "ref_sph")
    ref = os.path.join(ROOT, rel)
    impl = ("reference CUDA build, real = float (its src/config.h FP32 switch), sm_100a"
            if fp32 else "reference CUDA build, FP64, sm_100a, as shipped")
    line = {"impl": "reference", "metric": wl.metric, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if fp32 else "f64",
            "data": "synthetic",
            "config": {"workload": wl.name, "precision": args.precision,
                       "implementation": impl}}
    if not os.path.exists(ref):
        line["unavailable"] = "reference build %s is missing (build() compiles it)" % rel
        print(json.dumps(line))
        return 0
    with tempfile.TemporaryDirectory() as wd:
        wl.write(wd)
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
            r = subprocess.run([ref, "time", str(args.steps), str(args.warmup)], cwd=wd,
                               capture_output=True, text=True, timeout=3600)
        if r.returncode != 0:
            line["unavailable"] = "reference build failed: rc %d %s" % (r.returncode, r.stderr[-200:])
            print(json.dumps(line))
            return 0
        res = json.loads(r.stdout.strip().splitlines()[-1])
    sec = res["event_s"]
    value = res["N"] * args.steps / sec
    line.update(value=value, ms_per_step=1e3 * sec / args.steps,
                cpu_baseline={"value": value, "unit": UNIT, "cores": None, "kind": "reference",
                              "device": "cuda",
                              "sample": "the reference's own CUDA implementation of the step "
                                        "(it has no CPU path) on this GPU: %d timed steps after %d "
                                        "warm-up steps, CUDA events around the loop"
                                        % (args.steps, args.warmup)},
                e2e={"value": res["N"] * args.steps / res["wall_s"], "unit": UNIT,
                     "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                clocks=clk.summary(), gpu_launches=None)
    line["config"]["particles"] = res["N"]
    print(json.dumps(line))
    return 0


def run_ours(args, world, rank, local, dist, wl):
    import sph_b200

    with tempfile.TemporaryDirectory() as wd:
        path = wl.write(wd, args.lattice)
        pp = particles_file(path)
        sysm = sph_b200.System(path, [pp] if pp else None, precision=args.precision,
                               device=local)
        n = sysm.N
        tuning = sysm.autotune() if not args.no_autotune else sysm.tuning()
        sysm.step(args.warmup)
        sysm.synchronize()
        if dist is not None:
            dist.barrier()
        l0 = sysm.kernel_launches()
        with ClockSampler(local) as clk:
            sysm.step(args.steps)
            sysm.synchronize()
        ms = sysm.last_step_ms()
        launches = sysm.kernel_launches() - l0
        if dist is not None:
            dist.barrier()
        ms_max = max_over_ranks(dist, ms, local)
        value = n * args.steps * world / (ms_max * 1e-3)
        # per-phase device times (CUDA events on the engine's stream), separate short pass
        phases = sysm.profile_phases(args.profile_steps)
        # e2e: the reference's call sequence through the C ABI with host buffers; the step's
        # input (the magnetic moment) is copied from pinned host memory
        import torch

        m = torch.zeros(3, dtype=torch.float64).pin_memory().numpy()
        ke = []
        e2e_steps = min(args.steps, args.e2e_steps)
        info = sysm.info()
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            step = info["step"] + k + 1
            ang = info["omega_magnet"] * (info["t0"] + info["dt"] * step)
            m[0], m[1] = np.cos(ang), np.sin(ang)
            sysm.V_Verlet_step1()
            sysm.neighbours_search()
            sysm.calculate_forces(m)
            sysm.V_Verlet_step2()
            wf = sysm.wall_forces()
            ke.append(float(sysm.kinetic_energy()[0]) + 0.0 * float(wf[0, 0, 0]))
        e2e_dt = time.perf_counter() - t0
        e2e_dt = max_over_ranks(dist, e2e_dt, local)
        sysm.close()
    if rank != 0:
        return 0
    hbm, peak_kind = peaks()
    pair_ms = phases["pairs"]
    achieved = B_ALG_PAIRS[args.precision] * n / (pair_ms * 1e-3) / 1e9
    step_gbs = B_ALG_STEP[args.precision] * n * args.steps / (ms * 1e-3) / 1e9
    line = {
        "metric": wl.metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 pairs / f64 state",
        "data": ("synthetic (lattice, fluid velocities seeded uniform in +-1e-3 c, seed %d)" % SEED
                 if wl.key == "couette3d" else
                 "synthetic (lattice at rest, seeded colloid centres)"),
        "config": {"workload": wl.name, "particles": n, "precision": args.precision,
                   "parallelism": "replicas only" if world > 1 else "single box",
                   "launch_geometry": tuning,
                   "l2": "inputs larger than L2 (state ~0.7 GB > 126 MB), no flush",
                   "timing": "CUDA events around sph_step(K) on the engine stream, max over ranks"},
        "roofline": {"kernel": "k_pairs (fused velocity gradient, forces, dc/dt)",
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": args.pairs_traffic,
                     "note": "pair kernel is FP64/FP32-pipe bound (see profiles/); the HBM "
                             "fraction is reported as the metric asks"},
        "hbm_frac_step": step_gbs / hbm,
        "phase_ms": phases,
        "roofline_fp64": None if (args.precision != "fp64" or wl.key != "couette3d") else {
            "kernel": "k_pairs", "bound": "fp64",
            "achieved": FP64_PAIR_FLOP * n / (pair_ms * 1e-3) / 1e12,
            "peak": FP64_LANES * 2 * clock_mhz() * 1e6 / 1e12, "unit": "TFLOP/s",
            "frac": FP64_PAIR_FLOP * n / (pair_ms * 1e-3) / (FP64_LANES * 2 * clock_mhz() * 1e6),
            "note": "executed FP64 FLOP per particle counted by ncu (DADD + DMUL + 2 DFMA) over "
                    "the event-timed pair pass; peak = 9,472 FP64 FMA lanes x 2 x SM clock"},
        "e2e": {"value": n * e2e_steps / e2e_dt, "unit": UNIT, "h2d_bytes_per_step": 24,
                "d2h_bytes_per_step": 2 * 3 * 8 + 8, "steps": e2e_steps},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as wd:
            line["cpu_baseline"] = cpu_baseline(wd, wl, steps=1)
    if world == 1 and not args.no_secondary and wl.key == "couette3d" and args.lattice == 128:
        line["secondary"] = secondary_figures(args, local, wl)
    print(json.dumps(line))
    return 0


def mixed_summary(args, local, wl, steps=10, cmp_steps=5):
    """The same workload in mixed precision (pair terms in float, summed in FP64, state in
    FP64): device time per step, and its deviation from the FP64
    engine after cmp_steps steps from the same start (max |mixed - fp64| / group scale)."""
    import sph_b200

    # field groups: positions and c on their natural scale 1, the rest on the group's largest
    # FP64 magnitude
    groups = {"pos": (["x", "y", "z"], 1.0), "vel": (["vx", "vy", "vz"], None),
              "dens": (["dens"], None), "force": (["fx", "fy", "fz"], None),
              "conf": (["cxx", "cxy", "cyy", "cxz", "cyz", "czz"], 1.0),
              "dcdt": (["dcdt_xx", "dcdt_xy", "dcdt_yy", "dcdt_xz", "dcdt_yz", "dcdt_zz"], None)}

    def group_error(get_a, get_b, fields, scale):
        a = np.concatenate([get_a(f) for f in fields])
        b = np.concatenate([get_b(f) for f in fields])
        sc = scale if scale else max(float(np.abs(b).max()), 1e-300)
        return float(np.abs(a - b).max() / sc)

    with tempfile.TemporaryDirectory() as wd:
        path = wl.write(wd, args.lattice)
        pp = particles_file(path)
        b = sph_b200.System(path, [pp] if pp else None, precision="mixed", device=local)
        a = sph_b200.System(path, [pp] if pp else None, precision="fp64", device=local)
        a.step(cmp_steps)
        b.step(cmp_steps)
        a.synchronize()
        b.synchronize()
        errs = {g: group_error(b.field, a.field, f, sc) for g, (f, sc) in groups.items()}
        wa, wb = a.wall_forces(), b.wall_forces()
        errs["walls"] = float(np.abs(wa - wb).max() / np.abs(wa).max())
        a.close()
        b.step(3)
        b.synchronize()
        b.step(steps)
        b.synchronize()
        ms = b.last_step_ms() / steps
        n = b.N
        b.close()
    return {"precision": "mixed", "ms_per_step": ms, "value": n / (ms * 1e-3), "unit": UNIT,
            "steps": steps, "error_vs_fp64_after_%d_steps" % cmp_steps: errs,
            "timing": "CUDA events around sph_step(%d) after 3 warm-up steps" % steps}


def secondary_figures(args, local, wl):
    """Short measurements of the other workloads, recorded beside the headline: the mixed-
    precision engine on this workload, the 512-box batched ensemble against the same boxes
    run one at a time, and the surrogate's training throughput."""
    out = {}
    t0 = time.perf_counter()
    out["mixed_precision_128"] = mixed_summary(args, local, wl)
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.e2e_steps, sub.precision = 10, 3, 3, "fp64"
    ens = run_ensemble(sub, 1, 0, local, None, emit=False)
    out["ensemble512_fp64"] = {k: ens[k] for k in ("value", "unit", "ms_per_step", "steps",
                                                    "looped_single_box", "batched_over_looped")
                               if k in ens}
    sub.steps, sub.warmup = 200, 20
    sur = run_surrogate_train(sub, 1, 0, local, None, emit=False)
    out["surrogate_training"] = {k: sur[k] for k in ("metric", "value", "unit", "ms_per_step",
                                                      "steps", "roofline") if k in sur}
    out["seconds"] = time.perf_counter() - t0
    return out


ENSEMBLE_NAME = ("ensemble512: 512 independent 2D wall-bounded Oldroyd-B boxes with rotating "
                 "magnetic colloids, side 32..128 (sph_ensemble.draw_points seed 0)")


def timed_single_box(sph_b200, path, precision, device, steps, warmup=3):
    """Device time (ms) of `steps` steps of one box alone, after warm-up."""
    s = sph_b200.System(path, precision=precision, device=device)
    s.step(warmup)
    s.synchronize()
    s.step(steps)
    s.synchronize()
    ms, n = s.last_step_ms(), s.N
    s.close()
    return ms, n


def run_ensemble(args, world, rank, local, dist, emit=True):
    """The batched workload: 512 boxes advanced together in one context per GPU (boxes
    sharded over ranks by particle-steps, no exchange during the run), against the same
    boxes run one at a time."""
    import sph_b200
    import sph_ensemble

    pts = sph_ensemble.draw_points(512, seed=0)
    specs = [sph_ensemble.box_spec(pt) for pt in pts]
    costs = [sph_ensemble.box_cost(s, 1) for s in specs]
    parts = sph_ensemble.shard(costs, world)
    mine = parts[rank]
    with tempfile.TemporaryDirectory() as wd:
        paths, _ = sph_ensemble.write_inputs([pts[b] for b in mine], wd)
        sysm = sph_b200.System(paths, precision=args.precision, device=local)
        n = sysm.N
        tuning = sysm.autotune() if not args.no_autotune else sysm.tuning()
        sysm.step(args.warmup)
        sysm.synchronize()
        if dist is not None:
            dist.barrier()
        l0 = sysm.kernel_launches()
        with ClockSampler(local) as clk:
            sysm.step(args.steps)
            sysm.synchronize()
        ms = sysm.last_step_ms()
        launches = sysm.kernel_launches() - l0
        if dist is not None:
            dist.barrier()
        ms_max = max_over_ranks(dist, ms, local)
        n_all = sum(sph_ensemble.box_cost(s, 1) for s in specs)
        value = n_all * args.steps / (ms_max * 1e-3)
        # per-phase device times of the same step launched phase by phase (CUDA events between
        # the phases): their sum against the graph-replayed step shows what the graph's launch
        # gaps cost
        phases = sysm.profile_phases(args.profile_steps)
        # e2e: every step one observables sample of every box, read back to the host
        e2e_steps = min(args.steps, args.e2e_steps)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            sysm.step(1)
            sysm.observe()
            obs, _ = sysm.observables()
        e2e_dt = max_over_ranks(dist, time.perf_counter() - t0, local)
        nb_mine = len(mine)
        sysm.close()
        looped = None
        if world == 1 and rank == 0:
            # the same boxes one at a time: every 16th box, extrapolated by particle-steps
            sample = list(range(0, len(mine), 16))
            t_ms, n_s = 0.0, 0
            for k in sample:
                ms_b, nb = timed_single_box(sph_b200, paths[k], args.precision, local, args.steps)
                t_ms += ms_b
                n_s += nb
            looped = {"value": n_s * args.steps / (t_ms * 1e-3), "unit": UNIT,
                      "sample": "%d of the 512 boxes (every 16th), each alone in its own "
                                "context, %d graph-replayed steps after 3 warm-up steps, CUDA "
                                "events" % (len(sample), args.steps)}
    if rank != 0:
        return 0
    line = {
        "metric": "particle-steps/s (batched ensemble of 512 2D boxes)", "value": value,
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 pairs / f64 state",
        "data": "synthetic (lattice initial state, seeded parameters and colloid positions)",
        "config": {"workload": ENSEMBLE_NAME, "boxes": 512, "particles": n_all,
                   "precision": args.precision,
                   "parallelism": ("%d boxes on this rank of %d (sharded by particle-steps)"
                                   % (nb_mine, world)) if world > 1 else "one context",
                   "launch_geometry": tuning,
                   "timing": "CUDA events around sph_step(K), max over ranks"},
        "e2e": {"value": n_all * e2e_steps / e2e_dt, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 512 * 4 * 8, "steps": e2e_steps},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "phase_ms": phases,
        "phase_sum_ms": sum(phases.values()),
    }
    if looped:
        line["looped_single_box"] = looped
        line["batched_over_looped"] = value / looped["value"]
    if emit:
        print(json.dumps(line))
        return 0
    return line


SWEEP_NAME = ("sweep: 2D wall-bounded Oldroyd-B boxes with magnetic colloids at side 64, six "
               "physical inputs sampled over the batched workload's ranges; observables "
               "averaged over the last 75 percent of {steps} steps")


def sweep_line(args, nsteps, ntrain, nquery, t_one, t_data, npts, t_train, t_pred, t_fallback,
               mean_te, route_te, Yte, Ytr, route_q):
    """The JSON line of the sweep benchmark (kept apart so that it is tested on the CPU)."""
    import sph_surrogate

    keep = ~route_te
    err_kept = sph_surrogate.relative_error(mean_te[keep, 0], Yte[keep, 0]) if keep.any() else None
    err_all = sph_surrogate.relative_error(mean_te[:, 0], Yte[:, 0])
    base = sph_surrogate.relative_error(np.full(len(Yte), Ytr[:, 0].mean()), Yte[:, 0])

    def per_hour(n, s):
        return 3600.0 * n / s if s > 0 else None

    sur_marginal = per_hour(nquery, t_pred + t_fallback)
    one = per_hour(1, float(np.mean(t_one)))
    return {
        "metric": "sweep points/h at <=1% wall-stress error (surrogate with solver fallback)",
        "value": sur_marginal, "unit": "points/h", "n_gpus": 1, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "bf16 network / " + args.precision,
        "data": "synthetic (seeded sweep points)",
        "config": {"workload": SWEEP_NAME.format(steps=nsteps), "train_points": ntrain,
                   "heldout": len(Yte), "queries": nquery, "heads": 5,
                   "train_steps": args.sweep_train_steps, "batch": 1024, "route_tol": 0.02},
        "one_at_a_time_points_per_h": one,
        "batched_points_per_h": per_hour(npts, t_data),
        "surrogate_points_per_h_incl_data_and_training":
            per_hour(nquery, t_data + t_train + t_pred + t_fallback),
        "over_one_at_a_time": sur_marginal / one if sur_marginal and one else None,
        "heldout_wall_stress_error": {"unrouted": err_kept, "all": err_all,
                                      "mean_predictor": base, "measure": "mean |pred - true| / "
                                      "mean |true| over held-out points re-solved by the solver"},
        "heldout_errors_all_targets": [sph_surrogate.relative_error(mean_te[:, k], Yte[:, k])
                                       for k in range(4)],
        "routed_fraction": float(np.mean(route_q)),
        "seconds": {"one_point_mean": float(np.mean(t_one)), "training_data": t_data,
                    "training": t_train, "predict": t_pred, "fallback": t_fallback},
        "accepted": bool(err_kept is not None and err_kept <= 0.01),
    }


def run_sweep_bench(args, world, rank, local, dist):
    """Sweep points per hour: one-at-a-time plain runs, the batched solver, and the batched
    solver plus the surrogate (routing the points where its heads disagree back to the
    solver), with the surrogate's error on held-out points re-solved by the solver."""
    import sph_b200
    import sph_ensemble
    import sph_surrogate

    if world > 1 and rank != 0:
        return 0
    nsteps, ntrain, nquery = args.sweep_steps, args.sweep_train, 65536
    pts = sph_ensemble.draw_points(ntrain + 512, seed=1, fixed_N=64, coll_seed=7)
    queries = sph_ensemble.draw_points(nquery, seed=2, fixed_N=64, coll_seed=7)
    # the plain method one point at a time (a sample, each in its own context)
    t_one = []
    with tempfile.TemporaryDirectory() as wd:
        paths, _ = sph_ensemble.write_inputs(pts[:8], wd, nsteps=nsteps)
        for p in paths:
            t0 = time.perf_counter()
            s = sph_b200.System(p, precision=args.precision, device=local)
            sph_ensemble.run_sweep(s, nsteps, 20, warm=nsteps // 4)
            s.close()
            t_one.append(time.perf_counter() - t0)
    # the batched solver: training data and held-out points
    Y, t_data = sph_surrogate.solve_points(pts, nsteps, args.precision, local)
    X = sph_surrogate.features_of(pts)
    Xtr, Ytr, Xte, Yte = X[:ntrain], Y[:ntrain], X[ntrain:], Y[ntrain:]
    sur = sph_surrogate.Surrogate(heads=5, seed=0, device=local)
    t0 = time.perf_counter()
    sur.fit(Xtr, Ytr, steps=args.sweep_train_steps, lr=1e-3)
    t_train = time.perf_counter() - t0
    mean_te, route_te = sur.predict(Xte)
    # 65,536 queries: predicted, the disagreeing ones re-solved
    Xq = sph_surrogate.features_of(queries)
    t0 = time.perf_counter()
    mean_q, route_q = sur.predict(Xq)
    t_pred = time.perf_counter() - t0
    routed = [queries[k] for k in np.nonzero(route_q)[0]]
    _, t_fallback = sph_surrogate.solve_points(routed, nsteps, args.precision, local) if routed \
        else (None, 0.0)
    line = sweep_line(args, nsteps, ntrain, nquery, t_one, t_data, len(pts), t_train, t_pred,
                      t_fallback, mean_te, route_te, Yte, Ytr, route_q)
    print(json.dumps(line))
    return 0


def run_surrogate_train(args, world, rank, local, dist, emit=True):
    """Training throughput of the surrogate network (5 heads, batch 1024) on its tensor-core
    kernels: samples per second and the dense FLOP rate of the training step."""
    import torch

    import sph_surrogate

    if world > 1 and rank != 0:
        return 0
    heads, B = 5, 1024
    net = sph_surrogate.MLP(heads=heads, max_batch=B, seed=0, device=local)
    g = torch.Generator(device="cuda:%d" % local).manual_seed(0)
    x = torch.randn(B, 6, generator=g, device="cuda:%d" % local)
    y = torch.randn(B, 4, generator=g, device="cuda:%d" % local)
    for _ in range(args.warmup):
        net.train_step(x, y, 1e-3)
    net.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()  # the network runs on the legacy default stream, as torch does here
        for _ in range(args.steps):
            net.train_step(x, y, 1e-3)
        e1.record()
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    # multiply-adds per sample and head: forward 6*256 + 2*256*256 + 256*4; the backward
    # pass twice that (input and weight gradients), the 6-wide input gradient excepted
    fwd = 6 * 256 + 2 * 256 * 256 + 256 * 4
    flops = 2.0 * 3 * fwd * B * heads * args.steps
    tf = flops / (ms * 1e-3) / 1e12
    peak = None
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            peak = float(json.load(f).get("bf16_tflops", 0.0)) or None
    line = {"metric": "surrogate training samples/s (5 heads, batch 1024)",
            "value": B * args.steps / (ms * 1e-3), "unit": "samples/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 (fp32 accumulate)", "data": "synthetic",
            "config": {"workload": "surrogate network 6-256-256-256-4, 5 heads, Adam"},
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                         "frac": tf / peak if peak else None, "traffic": None,
                         "note": "1024 x 256 x 256 GEMMs: a step is a few microseconds of "
                                 "tensor work and is launch- and latency-bound"},
            "clocks": clk.summary()}
    net.close()
    if emit:
        print(json.dumps(line))
        return 0
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--sweep-steps", type=int, default=2000)
    ap.add_argument("--sweep-train", type=int, default=20480)
    ap.add_argument("--sweep-train-steps", type=int, default=3000)
    ap.add_argument("--workload", default="couette3d",
                    choices=["couette3d", "suspension96", "ensemble512", "sweep", "surrogate"],
                    help="couette3d: the headline 128^3 box; suspension96: the 96^3 box with 32 "
                         "magnetic colloids; ensemble512: 512 batched boxes; sweep: sweep "
                         "points per hour with the surrogate; surrogate: the network's "
                         "training throughput")
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="default: fp64 (the reference's precision); mixed for --workload sweep")
    ap.add_argument("--profile-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--pairs-traffic", type=float, default=None,
                    help="ncu DRAM bytes per k_pairs launch (default: the FP64 capture at "
                         "96^3, 505.8 MB, scaled by particle count to the benchmark)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the short mixed-precision, ensemble and surrogate figures that "
                         "the default couette3d line carries under 'secondary'")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch geometry (profiling runs: no tuning launches)")
    ap.add_argument("--lattice", type=int, default=None,
                    help="lattice side; the workload's own (128 for couette3d, 96 for "
                         "suspension96) is the benchmark, smaller sizes only for ncu captures")
    args = ap.parse_args()
    wl = WORKLOADS.get(args.workload)
    if wl is not None:
        if args.lattice is None:
            args.lattice = wl.lattice
        if args.lattice != wl.lattice:
            wl = Workload(wl.key, "%s_%d (profiling size, not the benchmark)" % (wl.key, args.lattice),
                          wl.metric, wl.write, args.lattice)
            args.no_cpu_baseline = True
    if (args.pairs_traffic is None and args.workload == "couette3d" and args.lattice == 128
            and args.precision in (None, "fp64")):
        # dram__bytes_read.sum + dram__bytes_write.sum of one k_pairs launch at 96^3
        # (940,032 particles), scaled to the 2,195,456 particles of the benchmark
        args.pairs_traffic = (386.815232e6 + 118.972928e6) * 2195456 / 940032
    if args.precision is None:
        args.precision = "mixed" if args.workload == "sweep" else "fp64"
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, dist = dist_setup(args)
    try:
        if args.workload == "surrogate":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable":
                                      "the reference has no learned component"}))
                return 0
            return run_surrogate_train(args, world, rank, local, dist)
        if args.workload == "sweep":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable":
                                      "the reference has no batched solver or surrogate; its "
                                      "one-box figure is the couette3d reference arm"}))
                return 0
            return run_sweep_bench(args, world, rank, local, dist)
        if args.workload == "ensemble512":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable":
                                      "the reference runs one box per process; its looped "
                                      "single-box figure is the couette3d reference arm"}))
                return 0
            return run_ensemble(args, world, rank, local, dist)
        if args.impl == "reference":
            return run_reference(args, world, rank, dist, wl)
        return run_ours(args, world, rank, local, dist, wl)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
