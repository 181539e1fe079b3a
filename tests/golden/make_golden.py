"""Generate the golden fixtures of tests/golden/ from the reference program itself.

Runs oracle/_ref/ref_sph -- the reference's own CUDA sources, compiled unmodified by
oracle/Makefile and driven by oracle/ref_harness.cu -- on small seeded configurations
and stores its state after the initial forces (step 0) and after a few steps as
compressed .npz files.  Needs a CUDA GPU (run it on the GPU machine):

    python tests/golden/make_golden.py [outdir [case ...]]

(with case names, only those fixtures are written).

The same configurations are defined in CASES and are read back by tests/test_golden.py,
which checks the CPU oracle against them.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "sph-magnetic-particles-oldroyd-b-in-cuda_b200"))
import oracle  # noqa: E402
import sph_input  # noqa: E402

STEPS = [0, 1, 5]
# cases stored at other steps
CASE_STEPS = {"kolmogorov64": [0, 1, 2000]}


def steps_of(name):
    return CASE_STEPS.get(name, STEPS)


def restart_3d_walls(workdir, seed=7):
    """16^3 walls box started from seeded random velocities through new_sim = 1."""
    base = dict(N=(16, 16, 16), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1,
                Vwall_bottom=-0.5, Vwall_top=0.5, dt=2e-5)
    p0 = os.path.join(workdir, "input_lattice")
    sph_input.write_input(p0, **base)
    o = oracle.Oracle(p0)
    n = o.info()["N"]
    rng = np.random.default_rng(seed)
    v = rng.uniform(-0.01, 0.01, size=(3, n))
    t = o.ifield("type")
    v[:, t != 0] = 0.0
    sph_input.write_particles(os.path.join(workdir, "input_particles.in"), 3,
                              o.field("x"), o.field("y"), o.field("z"), v[0], v[1], v[2],
                              o.field("mass"), t, o.field("cxx"), o.field("cxy"),
                              o.field("cyy"), o.field("cxz"), o.field("cyz"), o.field("czz"))
    o.close()
    return dict(base, new_sim=1)


CASES = {
    # 2D Kolmogorov flow (the reference's CPU-runnable configuration, reduced to 32^2)
    "kolmogorov2d": dict(N=(32, 32), L=(1.0, 1.0), dim=2, overlap=4.0, ext_force_type=2,
                         ext_force=(1.0, 0.0), dt=5e-5),
    # the reference's CPU-runnable configuration itself: 2D Kolmogorov flow, 64^2 particles,
    # stored after the initial forces, 1 step and its full length of 2000 steps
    "kolmogorov64": dict(N=(64, 64), L=(1.0, 1.0), dim=2, overlap=4.0, ext_force_type=2,
                         ext_force=(1.0, 0.0), dt=5e-5),
    # 2D Couette flow between y-walls
    "couette2d": dict(N=(32, 32), L=(1.0, 1.0), dim=2, overlap=3.0, wall=1,
                      Vwall_bottom=-0.5, Vwall_top=0.5, dt=2e-5),
    # 3D Couette flow from seeded velocities (restart file)
    "couette3d": "restart_3d_walls",
    # 2D walls + 3 magnetic colloids (repulsion, rotating dipole force, rigid bodies)
    "colloids2d": dict(N=(64, 64), L=(1.0, 1.0), dim=2, overlap=3.0, wall=1,
                       Vwall_bottom=-0.2, Vwall_top=0.2, dt=2e-5, N_colloids=3,
                       coll_R=4.0 / 64, coll_rho=1.0,
                       coll_x=((0.30, 0.50), (0.44, 0.52), (0.70, 0.35)),
                       coll_repulsion_cuton=0.05 * 4.0 / 64, F0_repulsion=1e-3,
                       tau_repulsion=2.0, cutoff_magnetic=0.3, F0_magnetic=1e-4,
                       omega_magnetic=6.2831853, ext_force_type=1, ext_force=(0.5, 0.0)),
    # 3D periodic box with 2 colloids (quaternion rotation, 3D magnetic |e| = R)
    "colloids3d": dict(N=(32, 32, 32), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, dt=2e-5,
                       N_colloids=2, coll_R=3.0 / 32, coll_rho=1.0,
                       coll_x=((0.41, 0.47, 0.52), (0.62, 0.51, 0.49)),
                       coll_repulsion_cuton=0.05 * 3.0 / 32, F0_repulsion=1e-3,
                       tau_repulsion=4.0, cutoff_magnetic=0.3, F0_magnetic=1e-3,
                       omega_magnetic=6.2831853),
}


# Cases whose fixtures are written by the reference build but not yet read by the tests
# (moved into CASES once their fixture is committed).
NEW_CASES = {}


DERIVED = ("gxx", "gxy", "gxz", "gyx", "gyy", "gyz", "gzx", "gzy", "gzz", "dcdt_xx",
           "dcdt_xy", "dcdt_yy", "dcdt_xz", "dcdt_yz", "dcdt_zz")


def keep(name, step, field):
    """Fields stored in the fixture.  Gradients and dc/dt are kept at step 0 only (later
    states carry them through c and v).  In the 3D colloid case they are not kept at all:
    the reference's 3D colloid gradient branch writes past a two-element array
    (src/kernel_vel_gradients.cu:463-466, 567-570), so its values are undefined."""
    if field in DERIVED and (step > 0 or name == "colloids3d"):
        return False
    if field in ("mass", "type") and step > 0:
        return False
    return True


def case_dir(name, workdir):
    """Write the input files of a case into workdir; returns the input dict."""
    spec = CASES[name] if name in CASES else NEW_CASES[name]
    if spec == "restart_3d_walls":
        spec = restart_3d_walls(workdir)
    sph_input.write_input(os.path.join(workdir, "input"), **spec)
    return spec


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden")
    names = sys.argv[2:] or list(CASES)
    os.makedirs(outdir, exist_ok=True)
    runs = os.path.join(outdir, "ref_runs.json")
    summary = json.load(open(runs)) if os.path.exists(runs) else {}
    for name in names:
        steps = steps_of(name)
        with tempfile.TemporaryDirectory() as wd:
            case_dir(name, wd)
            dump = os.path.join(wd, "dump")
            r = subprocess.run([oracle.REF_BIN, "dump", dump, ",".join(map(str, steps))],
                               cwd=wd, capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                raise RuntimeError("%s: ref_sph failed (%d): %s %s" % (name, r.returncode,
                                                                       r.stdout[-400:], r.stderr[-400:]))
            arrays = {}
            for s in steps:
                d = oracle.read_ref_dump(os.path.join(dump, "ref_step%06d.bin" % s))
                for k, v in d.items():
                    if keep(name, s, k):
                        arrays["s%d_%s" % (s, k)] = v
            np.savez_compressed(os.path.join(outdir, name + ".npz"), **arrays)
            summary[name] = r.stdout.strip()
            print(name, r.stdout.strip())
    with open(runs, "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
