"""Parameter sweeps over ensembles of independent 2D wall-bounded boxes.

A sweep point is one box: a Couette cell of side N lattice spacings (L = 1, overlap 4,
walls normal to y moving at +-Vwall) filled with an Oldroyd-B fluid of relaxation time tau
and polymer modulus nkT, holding up to 24 magnetic colloids (R = 4 dx) in a field
rotating at omega.  `draw_points` samples the parameter space, `box_spec` turns one point
into the keys of a reference `input` file, and `run_sweep` advances a whole batch in one
engine context (one launch per step phase for all boxes, the step replayed as a CUDA
graph) and returns every box's time-averaged observables.

Rules where the sampled corners are not feasible as stated (kept deterministic per seed):
  * colloid coarse grid: the reference needs at least 3 coarse cells per axis, i.e. the
    larger of the repulsion reach 2R + 5R/tau_rep and the magnetic cutoff at most L/3
    (system_initialize.cpp:225-247).  Per box the magnetic cutoff is min(6R, 0.33) and
    tau_repulsion = max(1, 5R / (0.33 - 2R)).
  * colloid count: positions are drawn uniformly with centre distances >= 2.2 R (periodic
    in x) and at least R + rcut from the walls; a colloid that finds no place in 2000
    draws ends the placement, so the count is capped by what fits.
"""
import math
import os

import numpy as np

import sph_input

# the six inputs of a sweep point (the surrogate's features)
FEATURES = ["Wi", "omega_tau", "phi", "F0_ratio", "Vwall", "nkT"]
# fixed physics of the sweep (unspecified by the workload; the plain method's values)
FIXED = dict(dt=2e-5, eta=0.1, c=10.0, P0=0.0, rho=1.0, zeta=0.0, kT=0.01, F0_repulsion=1e-3)


def draw_points(n, seed=0, fixed_N=None, coll_seed=None):
    """n sweep points: dicts with the box side N and the sampled physical parameters.
    fixed_N and coll_seed pin the resolution and the colloid placement sequence (the
    first k colloids of every point then sit at the same places), which makes the
    observables functions of the six physical inputs alone (the surrogate's sweeps)."""
    rng = np.random.default_rng(seed)
    pts = []
    for _ in range(n):
        N = int(rng.integers(32, 129))
        pts.append(dict(
            N=int(fixed_N) if fixed_N else N,
            tau=float(10 ** rng.uniform(-1, 1)),
            omega_tau=float(10 ** rng.uniform(-1, 1)),
            ncoll=int(rng.integers(0, 25)),
            F0_ratio=float(rng.uniform(0.1, 2.0)),
            Vwall=float(rng.uniform(0.1, 1.0)),
            nkT=float(rng.uniform(0.5, 2.0)),
            seed=int(rng.integers(0, 2 ** 31 - 1)),
        ))
        if coll_seed is not None:
            pts[-1]["seed"] = int(coll_seed)
    return pts


def place_colloids(n, R, rcut, seed):
    """Up to n centres in the unit box, >= 2.2 R apart (periodic in x), clear of the walls."""
    rng = np.random.default_rng(seed)
    lo, hi = R + rcut, 1.0 - R - rcut
    out = []
    for _ in range(n):
        for _ in range(2000):
            x, y = float(rng.uniform(0.0, 1.0)), float(rng.uniform(lo, hi))
            ok = True
            for (a, b) in out:
                dx = x - a
                dx -= round(dx)
                if dx * dx + (y - b) ** 2 < (2.2 * R) ** 2:
                    ok = False
                    break
            if ok:
                out.append((x, y))
                break
        else:
            break
    return out


def box_spec(pt, nsteps=5000):
    """The `input` keys of one sweep point (see the module notes for the rules)."""
    N = pt["N"]
    dx = 1.0 / N
    R = 4.0 * dx
    rcut = 4.0 * dx
    coll = place_colloids(pt["ncoll"], R, rcut, pt["seed"])
    tau_rep = max(1.0, 5.0 * R / (0.33 - 2.0 * R))
    spec = dict(
        N=(N, N), L=(1.0, 1.0), dim=2, overlap=4.0, wall=1, Nsteps=nsteps,
        Vwall_top=pt["Vwall"], Vwall_bottom=-pt["Vwall"], tau=pt["tau"],
        np=pt["nkT"] / FIXED["kT"], kT=FIXED["kT"], dt=FIXED["dt"], eta=FIXED["eta"],
        c=FIXED["c"], P0=FIXED["P0"], rho=FIXED["rho"], zeta=FIXED["zeta"],
        N_colloids=len(coll), coll_R=R, coll_rho=1.0, coll_move=1, coll_x=tuple(coll),
        coll_repulsion_cuton=0.05 * R, F0_repulsion=FIXED["F0_repulsion"],
        tau_repulsion=tau_rep, cutoff_magnetic=min(6.0 * R, 0.33),
        F0_magnetic=pt["F0_ratio"] * FIXED["F0_repulsion"],
        omega_magnetic=pt["omega_tau"] / pt["tau"],
    )
    return spec


def features(pt, spec):
    """The surrogate's six inputs of a sweep point."""
    R = spec["coll_R"]
    return np.array([
        2.0 * pt["Vwall"] * pt["tau"],                # Weissenberg number tau * shear rate
        pt["omega_tau"],
        spec["N_colloids"] * math.pi * R * R,         # colloid area fraction (L = 1)
        pt["F0_ratio"],
        pt["Vwall"],
        pt["nkT"],
    ])


def write_inputs(pts, workdir, nsteps=5000):
    """Write one `input` file per point; returns the paths and the specs."""
    os.makedirs(workdir, exist_ok=True)
    paths, specs = [], []
    for k, pt in enumerate(pts):
        spec = box_spec(pt, nsteps)
        p = os.path.join(workdir, "input_%05d" % k)
        sph_input.write_input(p, **spec)
        paths.append(p)
        specs.append(spec)
    return paths, specs


def box_cost(spec, nsteps=None):
    """Cost estimate of a box: particles x steps (the lattice plus the wall layers)."""
    N = spec["N"]
    rows = N[1] + (2 * int(math.ceil(spec["overlap"])) if spec.get("wall", 0) else 0)
    n = N[0] * rows * (N[2] if spec.get("dim", 2) == 3 else 1)
    return n * (nsteps if nsteps is not None else spec.get("Nsteps", 1))


def shard(costs, world):
    """Partition boxes over `world` ranks by cost (longest first onto the least loaded
    rank); ranks are independent, no exchange during the run.  Returns one sorted list of
    box indices per rank."""
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for b in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(b)
        loads[r] += costs[b]
    return [sorted(p) for p in parts]


def gather_by_box(dist, parts, rank, local_rows, nboxes):
    """Collect every rank's per-box result rows (local_rows[k] belongs to box
    parts[rank][k]) into one nboxes-long list in box order, on every rank.  dist is
    torch.distributed (any backend) or None for one rank."""
    if dist is None:
        gathered = [list(local_rows)]
    else:
        gathered = [None] * dist.get_world_size()
        dist.all_gather_object(gathered, list(local_rows))
    out = [None] * nboxes
    for r, rows in enumerate(gathered):
        for b, row in zip(parts[r], rows):
            out[b] = row
    assert all(x is not None for x in out), "a box was not run"
    return out


def run_sweep(system, nsteps, observe_every=10, warm=0):
    """Advance every box of `system` (an sph_b200.System over the batch) by nsteps and
    return (nboxes x 4 observables averaged over the samples after `warm` steps, samples)."""
    done = 0
    if warm:
        system.step(warm)
        done = warm
    system.reset_observables()
    while done < nsteps:
        k = min(observe_every, nsteps - done)
        system.step(k)
        system.observe()
        done += k
    return system.observables()
