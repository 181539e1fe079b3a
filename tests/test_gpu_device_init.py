"""Device-side initialisation (sph_options.init_on_device): lattice boxes built on the GPU
give the same bits as the host set-up (system_initialize_particles_new_sim.cpp:21-140,
system_initialize.cpp:277-355) -- initial state, per-box counts and every field after
steps.  Restart boxes and colloid shells stay on the host inside the same context."""
import os

import numpy as np
import pytest

import make_golden as mg
import sph_b200
import sph_ensemble

pytestmark = pytest.mark.gpu

STATE = ["x", "y", "z", "vx", "vy", "vz", "mass", "cxx", "cxy", "cyy", "cxz", "cyz", "czz"]
AFTER = ["x", "y", "z", "vx", "vy", "vz", "fx", "fy", "dens", "press", "cxx", "cxy", "cyy",
         "dcdt_xy"]
INFO = ["N", "Nmax", "Nlist_walls", "Nlist_colloids", "N_colloids"]


def assert_same(a, b, label, steps=3):
    assert a.N == b.N, label
    for box in range(a.nboxes):
        ia, ib = a.info(box), b.info(box)
        for k in INFO:
            assert ia[k] == ib[k], (label, box, k, ia[k], ib[k])
    assert np.array_equal(a.type(), b.type()), label
    for f in STATE:
        assert np.array_equal(a.field(f), b.field(f)), (label, "initial", f)
    for f in sph_b200.COLLOID_FIELDS[:14]:
        assert np.array_equal(a.colloid_field(f), b.colloid_field(f)), (label, f)
    a.step(steps)
    b.step(steps)
    a.synchronize()
    b.synchronize()
    for f in AFTER:
        assert np.array_equal(a.field(f), b.field(f)), (label, "after", f)
    assert np.array_equal(a.wall_forces(), b.wall_forces()), label
    assert np.array_equal(a.kinetic_energy(), b.kinetic_energy()), label
    for f in sph_b200.COLLOID_FIELDS:
        assert np.array_equal(a.colloid_field(f), b.colloid_field(f)), (label, "after", f)


@pytest.mark.parametrize("name", list(mg.CASES))
def test_device_init_matches_host(name, workdir):
    """Every golden configuration: periodic and walled, 2D and 3D, colloids carved from
    the lattice (with shells) and the restart-file case (built on the host either way)."""
    mg.case_dir(name, workdir)
    pp = os.path.join(workdir, "input_particles.in")
    pp = [pp] if os.path.exists(pp) else None
    inp = os.path.join(workdir, "input")
    host = sph_b200.System(inp, pp, init_on_device=False)
    dev = sph_b200.System(inp, pp, init_on_device=True)
    assert_same(dev, host, name)
    dev.close()
    host.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_init_ensemble_matches_host(precision, workdir):
    """An ensemble of 24 boxes of uneven size with 0..24 colloids each."""
    pts = sph_ensemble.draw_points(24, seed=3)
    paths, _ = sph_ensemble.write_inputs(pts, workdir, nsteps=100)
    host = sph_b200.System(paths, precision=precision, init_on_device=False)
    dev = sph_b200.System(paths, precision=precision, init_on_device=True)
    assert_same(dev, host, "ensemble24", steps=4)
    dev.close()
    host.close()


def test_device_init_mixed_walled_and_periodic(workdir):
    """Walled and periodic boxes, with and without colloids, in one context: each lattice
    box lands at its own slots and walls-list entries."""
    import sph_input

    specs = [
        dict(N=(32, 32), L=(1.0, 1.0), dim=2, overlap=4.0, wall=1, Vwall_top=0.3,
             Vwall_bottom=-0.3, dt=2e-5),
        dict(N=(40, 40), L=(1.0, 1.0), dim=2, overlap=4.0, wall=0, ext_force_type=2,
             ext_force=(1.0, 0.0), dt=5e-5),
        dict(N=(48, 40), L=(1.2, 1.0), dim=2, overlap=4.0, wall=1, Vwall_top=0.1,
             Vwall_bottom=-0.1, dt=2e-5, tau=2.0, N_colloids=2, coll_R=4.0 / 40,
             coll_x=((0.3, 0.5), (0.8, 0.45)), tau_repulsion=5.0, cutoff_magnetic=0.3,
             F0_magnetic=1e-4, F0_repulsion=1e-3, omega_magnetic=3.0),
        dict(N=(36, 36), L=(1.0, 1.0), dim=2, overlap=4.0, wall=0, dt=2e-5, N_colloids=1,
             coll_R=4.0 / 36, coll_x=((0.97, 0.03),), tau_repulsion=5.0, cutoff_magnetic=0.3,
             F0_magnetic=1e-4, F0_repulsion=1e-3, omega_magnetic=3.0),
        dict(N=(32, 32), L=(1.0, 1.0), dim=2, overlap=3.0, wall=1, Vwall_top=0.5,
             Vwall_bottom=-0.5, dt=2e-5),
    ]
    paths = []
    for k, spec in enumerate(specs):
        p = os.path.join(workdir, "input%d" % k)
        sph_input.write_input(p, **spec)
        paths.append(p)
    host = sph_b200.System(paths, init_on_device=False)
    dev = sph_b200.System(paths, init_on_device=True)
    assert_same(dev, host, "walled+periodic", steps=3)
    dev.close()
    host.close()


def test_device_init_periodic_colloids_3d(workdir):
    """Colloids near the periodic faces of a walled 3D box: the carving wraps in x and z
    (and not in y, where the walls are)."""
    import sph_input

    p = os.path.join(workdir, "input")
    R = 3.0 / 24
    sph_input.write_input(p, N=(24, 24, 24), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1,
                          Vwall_bottom=-0.1, Vwall_top=0.1, dt=2e-5, N_colloids=2, coll_R=R,
                          coll_rho=1.0, coll_x=((0.02, 0.5, 0.98), (0.6, 0.3, 0.5)),
                          tau_repulsion=10.0, cutoff_magnetic=0.3, F0_magnetic=1e-4,
                          F0_repulsion=1e-3, omega_magnetic=3.0)
    host = sph_b200.System(p, init_on_device=False)
    dev = sph_b200.System(p, init_on_device=True)
    assert_same(dev, host, "periodic3d", steps=2)
    dev.close()
    host.close()
