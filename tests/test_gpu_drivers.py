"""Drop-in check of the whole program: the reference's own driver (src/main.cu) re-linked
against the engine's class_system shim, and the engine's sph_run driver, write the same
output files as the reference's unmodified program on the same input.

Built by oracle/Makefile (targets ref_main and shim_main) and the engine's Makefile
(sph_run); the reference program runs on the GPU, so these are GPU tests."""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

import sph_input
from make_golden import CASES, restart_3d_walls

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ref_main")
SHIM_MAIN = os.path.join(ROOT, "oracle", "_ref", "shim_main")
SPH_RUN = os.path.join(ROOT, "sph-magnetic-particles-oldroyd-b-in-cuda_b200", "lib", "sph_run")

pytestmark = pytest.mark.gpu

# output cadence of the test runs (every kind of file at several steps)
OUT = dict(Nsteps=20, freq_micro=10, freq_macro=5, freq_walls=5, freq_colloids=5)


def write_case(name, wd):
    spec = CASES[name]
    if spec == "restart_3d_walls":
        spec = restart_3d_walls(wd)
    sph_input.write_input(os.path.join(wd, "input"), **dict(spec, **OUT))


def run(cmd, wd):
    r = subprocess.run(cmd, cwd=wd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (cmd, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def outputs(wd):
    return sorted(os.path.basename(p) for p in glob.glob(os.path.join(wd, "*.dat")))


def compare_file(a, b):
    """Same rows and columns; integer columns equal, real columns within the last printed
    digit (the engines agree to ~1e-12; an 8-decimal print may still round apart)."""
    ta = open(a).read().split("\n")
    tb = open(b).read().split("\n")
    assert len(ta) == len(tb), (a, len(ta), len(tb))
    worst = 0.0
    for la, lb in zip(ta, tb):
        fa, fb = la.split(), lb.split()
        assert len(fa) == len(fb), (a, la, lb)
        for x, y in zip(fa, fb):
            if "." not in y:
                assert x == y, (a, la, lb)
                continue
            u, v = float(x), float(y)
            d = abs(u - v)
            worst = max(worst, d)
            assert d <= 1.5e-8 + 1e-10 * abs(v) or (os.path.basename(a) == "macro.dat"
                                                     and d <= 1.5e-6), (a, la, lb)
    return worst


def need(path):
    if not os.path.exists(path):
        pytest.skip("%s is not built" % os.path.relpath(path, ROOT))


def setup_dirs(tmp_path, case, names):
    dirs = {k: tmp_path / k for k in names}
    for d in dirs.values():
        d.mkdir()
    first = dirs[names[0]]
    write_case(case, str(first))
    for k in names[1:]:
        for f in os.listdir(first):
            shutil.copy(first / f, dirs[k] / f)
    return dirs


def test_main_on_shim_and_sph_run_match_reference_program(tmp_path):
    """2D walls + magnetic colloids + body force: every output file of the reference's
    program, its main.cu on the shim, and sph_run, compared value by value."""
    need(REF_MAIN)
    need(SHIM_MAIN)
    need(SPH_RUN)
    dirs = setup_dirs(tmp_path, "colloids2d", ["ref", "shim", "run"])
    run([REF_MAIN], str(dirs["ref"]))
    run([SHIM_MAIN], str(dirs["shim"]))
    run([SPH_RUN, "--quiet"], str(dirs["run"]))
    ref_files = outputs(str(dirs["ref"]))
    assert {"macro.dat", "micro-0.dat", "micro-20.dat", "walls-5.dat",
            "colloids-20.dat"} <= set(ref_files)
    for k in ("shim", "run"):
        assert outputs(str(dirs[k])) == ref_files, k
        for f in ref_files:
            compare_file(str(dirs[k] / f), str(dirs["ref"] / f))


MICRO_COLS = {2: ["x", "y", "vx", "vy", "mass", "dens", "press", "type", "cxx", "cxy", "cyy"],
              3: ["x", "y", "z", "vx", "vy", "vz", "mass", "dens", "press", "type", "cxx", "cxy",
                  "cyy", "cxz", "cyz", "czz"]}


@pytest.mark.parametrize("case", ["kolmogorov2d", "couette3d"])
def test_main_on_shim_and_sph_run_without_colloids(tmp_path, case):
    """Boxes without colloids.  The reference's unmodified program writes nothing here:
    main.cu:278-281 copies the magnetic moment into a buffer that copy_pointers_to_device
    allocates only with colloids, and the next error check ends the run.  The shim clears
    that stale error, so its run goes on; its micro files and sph_run's are checked
    against the CPU oracle (itself pinned to the reference's kernels) at the same steps."""
    import oracle

    need(SHIM_MAIN)
    need(SPH_RUN)
    dirs = setup_dirs(tmp_path, case, ["shim", "run", "orc"])
    run([SHIM_MAIN], str(dirs["shim"]))
    run([SPH_RUN, "--quiet"], str(dirs["run"]))
    files = outputs(str(dirs["shim"]))
    assert outputs(str(dirs["run"])) == files
    assert {"macro.dat", "micro-0.dat", "micro-10.dat", "micro-20.dat"} <= set(files)
    for f in files:
        compare_file(str(dirs["run"] / f), str(dirs["shim"] / f))
    wd = str(dirs["orc"])
    particles = os.path.join(wd, "input_particles.in")
    o = oracle.Oracle(os.path.join(wd, "input"),
                      particles if os.path.exists(particles) else None)
    dim = o.info()["dim"]
    done = 0
    for step in (0, 10, 20):
        o.run(step - done)
        done = step
        table = np.loadtxt(str(dirs["shim"] / ("micro-%d.dat" % step)))
        assert np.array_equal(table[:, 0], np.arange(table.shape[0]))
        for c, name in enumerate(MICRO_COLS[dim], start=1):
            ref = o.ifield(name) if name == "type" else o.field(name)
            err = np.abs(table[:, c] - ref)
            assert np.all(err <= 1.5e-8 + 1e-10 * np.abs(ref)), (step, name, float(err.max()))
    o.close()


def test_sph_run_checkpoint_restart_is_bitwise(tmp_path):
    """20 steps in one go equal 10 steps, a binary checkpoint, and 10 more steps from it."""
    need(SPH_RUN)
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    write_case("colloids2d", str(a))
    for f in os.listdir(a):
        shutil.copy(a / f, b / f)
    run([SPH_RUN, "--quiet", "--steps", "20", "--checkpoint", "end.ckpt"], str(a))
    run([SPH_RUN, "--quiet", "--steps", "10", "--checkpoint", "mid.ckpt"], str(b))
    run([SPH_RUN, "--quiet", "--steps", "10", "--restart", "mid.ckpt", "--checkpoint",
         "end.ckpt"], str(b))
    assert open(a / "end.ckpt", "rb").read() == open(b / "end.ckpt", "rb").read()
    for f in ("micro-20.dat", "colloids-20.dat", "walls-20.dat"):
        assert open(a / f).read() == open(b / f).read(), f
