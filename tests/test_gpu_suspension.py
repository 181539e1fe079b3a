"""The 3D suspension of rotating magnetic colloids at its own size: 96^3 lattice between
walls at rest, 32 colloids of radius 4 dx (sph_input.suspension_spec, seeded centres).

It exercises, at scale, the 3D paths no smaller case reaches with this many colloids: the
quaternion update of the rigid bodies (kernel_move_colloids_VV_part1.cu:119-140), the 3D
magnetic force with its |e| = R scaling (kernel_magnetic_force_colloids.cu:181-184), the
repulsion with its r^2 clamp (kernel_repulsion_force_colloids.cu:108-121), the collected
forces and torques of 32 particle shells, and the wall forces.

FP64 engine against the FP64 oracle after the initial forces, 1 and 10 steps: every fluid
and colloid field group, the quaternions and the wall forces within 1e-10 (steps 0 and 1)
and 1e-9 (step 10) of their scale, integer cell and colloid-grid arrays bit-exact.  The
torque on every colloid is nonzero at step 0, so the 3D rotation never divides by a zero
angular velocity (kernel_move_colloids_VV_part1.cu:123-125 would give NaN).
"""
import os

import numpy as np
import pytest

import oracle
import sph_b200
import sph_input
from conftest import COLLOID_GROUPS, GROUPS, group_error

pytestmark = pytest.mark.gpu
INTS = ["particle_cell", "particle_index", "cell_start", "cell_end"]
CINTS = ["coll_cell", "coll_index", "coll_cell_start", "coll_cell_end"]


def compare(e, o, tol, label):
    errs = {}
    for gname, (fields, norm) in GROUPS.items():
        if gname == "grad":
            continue
        errs[gname] = group_error(e.field, o.field, fields, norm, 3)
    for gname, (fields, norm) in COLLOID_GROUPS.items():
        errs[gname] = group_error(e.colloid_field, o.field, fields, norm, 3)
    q = ["coll_quat0", "coll_quatx", "coll_quaty", "coll_quatz"]
    errs["quat"] = max(float(np.abs(e.colloid_field(k) - o.field(k)).max()) for k in q)
    wf = e.wall_forces()[0]
    ref = np.stack([o.field("fx_wall"), o.field("fy_wall"), o.field("fz_wall")], axis=1)
    errs["walls"] = float(np.abs(wf - ref).max() / np.abs(ref).max())
    for k, v in errs.items():
        assert v <= tol, (label, k, v)
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), (label, k)
    cc = e.export_colloid_cells()
    for k in CINTS:
        assert np.array_equal(cc[k], o.ifield(k)), (label, k)
    return errs


def test_suspension96_fp64_matches_oracle(workdir):
    spec = sph_input.suspension_spec()
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, **spec)
    oracle.set_threads(os.cpu_count() or 1)
    e = sph_b200.System(inp, precision="fp64")
    o = oracle.Oracle(inp)
    assert e.N == o.info()["N"] and e.ncoll == 32
    assert o.run(0) == 0
    e.step(0)
    compare(e, o, 1e-10, "step0")
    T = np.stack([e.colloid_field(k) for k in ["tx_colloid", "ty_colloid", "tz_colloid"]], 1)
    assert np.all(np.linalg.norm(T, axis=1) > 0.0)
    assert o.run(1) == 0
    e.step(1)
    e.synchronize()
    compare(e, o, 1e-10, "step1")
    assert o.run(9) == 0
    e.step(9)
    e.synchronize()
    errs = compare(e, o, 1e-9, "step10")
    assert e.info()["step"] == 10, errs
    e.close()
    o.close()


# Mixed precision against FP64 after the 2000 steps of the configuration, with the magnetic
# and repulsion amplitudes scaled by 1e-4 (F0_repulsion 1e-3, F0_magnetic 5e-4): as written
# (10 and 5) the colloids reach hundreds of box lengths per unit time and one leaves the box
# at step 154 (FP64 engine).  Bounds: about 3-10 times the errors measured on B200
# (positions 9e-8 of L, colloid positions 3e-8, quaternions 1.4e-8, colloid velocities
# 3.4e-6 and angular velocities 4.5e-6 of their scale, wall forces 1.6e-8, fluid velocities
# 1.3e-5, density 6e-6, conformation 7e-6, forces 7.5e-6; colloid forces 8.3e-5 and torques
# 9.4e-4, small residuals of large cancelling fluid forces).
TRAJ_TOL = dict(pos=1e-6, vel=2e-4, force=1e-4, dens=5e-5, press=5e-5, conf=1e-4, dcdt=5e-4,
                cpos=3e-7, cvel=5e-5, comega=5e-5, cforce=5e-4, ctorque=1e-2, quat=2e-7,
                walls=1e-6)


def test_suspension96_mixed_follows_fp64_for_2000_steps(workdir):
    spec = sph_input.suspension_spec(F0_repulsion=1e-3, F0_magnetic=5e-4)
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, **spec)
    a = sph_b200.System(inp, precision="fp64")
    b = sph_b200.System(inp, precision="mixed")
    a.step(2000)
    b.step(2000)
    a.synchronize()
    b.synchronize()
    assert a.info()["step"] == b.info()["step"] == 2000
    errs = {}
    for gname, (fields, norm) in GROUPS.items():
        if gname != "grad":
            errs[gname] = group_error(b.field, a.field, fields, norm, 3)
    for gname, (fields, norm) in COLLOID_GROUPS.items():
        errs[gname] = group_error(b.colloid_field, a.colloid_field, fields, norm, 3)
    q = ["coll_quat0", "coll_quatx", "coll_quaty", "coll_quatz"]
    errs["quat"] = max(float(np.abs(a.colloid_field(k) - b.colloid_field(k)).max()) for k in q)
    wa, wb = a.wall_forces(), b.wall_forces()
    errs["walls"] = float(np.abs(wa - wb).max() / np.abs(wa).max())
    for k, v in errs.items():
        assert v <= TRAJ_TOL[k], (k, v, errs)
    # the colloids stay in the box, clear of the walls
    y = a.colloid_field("coll_y")
    assert np.all(np.isfinite(y)) and y.min() > 0.0 and y.max() < 1.0
    a.close()
    b.close()
