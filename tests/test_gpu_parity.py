"""Parity of the CUDA engine (through its C ABI) with the FP64 oracle and with the
reference build's golden dumps.

Tolerances (max |engine - oracle| / scale of the field group, see conftest.GROUPS):
  FP64 engine  : 1e-10 for every group; integer cell / sort arrays bit-exact.
  mixed engine : pair arithmetic in float; states (positions, conformation tensor,
                 density, velocities) within 2e-5 and forces / dc/dt within 5e-5 after 5
                 steps.  Two quantities that are small residuals of large cancelling
                 float terms get a stated wider bound: forces and velocities of a fluid
                 at rest on a perfect lattice (Kolmogorov start, 5e-3) and colloid torques
                 and angular velocities (2e-3).
"""
import os

import numpy as np
import pytest

import make_golden as mg
import oracle
import sph_b200
import sph_input
from conftest import COLLOID_GROUPS, GROUPS, group_error

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
INTS = ["particle_cell", "particle_index", "cell_start", "cell_end"]

MIXED_TOL = dict(pos=1e-9, conf=1e-8, dens=2e-5, press=2e-5, vel=2e-5, force=5e-5, dcdt=5e-5,
                 grad=5e-5, cpos=1e-9, cvel=2e-5, comega=2e-3, cforce=5e-5, ctorque=2e-3,
                 walls=2e-5)
MIXED_WIDE = {"kolmogorov2d": dict(vel=5e-3, force=5e-3, dcdt=5e-3),
              # measured on B200 at step 5: forces 7.4e-3, dc/dt 1.2e-2 of their scales
              "kolmogorov64": dict(vel=5e-3, force=2e-2, dcdt=3e-2)}


def open_case(name, workdir, precision="fp64", use_graph=True):
    mg.case_dir(name, workdir)
    pp = os.path.join(workdir, "input_particles.in")
    pp = pp if os.path.exists(pp) else None
    inp = os.path.join(workdir, "input")
    e = sph_b200.System(inp, [pp] if pp else None, precision=precision, use_graph=use_graph)
    return e, oracle.Oracle(inp, pp)


def compare_state(e, o, tol, label, skip=()):
    dim = o.info()["dim"]
    errs = {}
    for gname, (fields, norm) in GROUPS.items():
        if gname in skip or gname == "grad":
            continue
        errs[gname] = group_error(e.field, o.field, fields, norm, dim)
    if o.info()["N_colloids"]:
        for gname, (fields, norm) in COLLOID_GROUPS.items():
            errs[gname] = group_error(e.colloid_field, o.field, fields, norm, dim)
    if o.info()["wall"]:
        wf = e.wall_forces()[0]
        ref = np.stack([o.field("fx_wall"), o.field("fy_wall"), o.field("fz_wall")], axis=1)
        if dim == 2:
            wf, ref = wf[:, :2], ref[:, :2]
        errs["walls"] = float(np.abs(wf - ref).max() / max(np.abs(ref).max(), 1e-300))
    for k, v in errs.items():
        t = tol if isinstance(tol, float) else tol[k]
        assert v <= t, (label, k, v, t)
    return errs


@pytest.mark.parametrize("name", list(mg.CASES))
def test_fp64_engine_matches_oracle(name, workdir):
    e, o = open_case(name, workdir)
    o.run(0)
    e.step(0)
    compare_state(e, o, 1e-10, "step0")
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), k
    o.run(5)
    e.step(5)
    e.synchronize()
    compare_state(e, o, 1e-10, "step5")
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), k
    if o.info()["N_colloids"] >= 2:
        cc = e.export_colloid_cells()
        for k in ["coll_cell", "coll_index", "coll_cell_start", "coll_cell_end"]:
            assert np.array_equal(cc[k], o.ifield(k)), k
    assert e.kernel_launches() > 0


LONG = {
    # config 1 at its own size and length: 2D Kolmogorov flow, 64^2 = 4,096 particles,
    # 2000 steps
    "kolmogorov64": (mg.CASES["kolmogorov64"], 2000),
    "couette2d": (mg.CASES["couette2d"], 100),
    "colloids2d": (mg.CASES["colloids2d"], 100),
    "colloids3d": (mg.CASES["colloids3d"], 30),
}


@pytest.mark.parametrize("name", list(LONG))
def test_fp64_engine_matches_oracle_after_n_steps(name, workdir):
    """FP64 engine against the FP64 oracle after N steps (the oracle is built without FMA
    contraction, the engine with it).  Tolerance 1e-9 of each field group's scale."""
    spec, nsteps = LONG[name]
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, **spec)
    e = sph_b200.System(inp)
    o = oracle.Oracle(inp)
    o.run(0)
    e.step(0)
    o.run(nsteps)
    e.step(nsteps)
    e.synchronize()
    errs = compare_state(e, o, 1e-9, "step%d" % nsteps)
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), k
    assert e.info()["step"] == nsteps, errs
    e.close()
    o.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_cells_match_oracle(precision, workdir):
    """A walled 3D box at overlap 4: cells of 64 particles, so the list build takes two
    rounds per cell and more chunks per neighbourhood walk than its mask table holds (the
    table is decoded part-way).  Against the FP64 oracle after 3 steps, cells bit-exact."""
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, N=(24, 24, 24), L=(1.0, 1.0, 1.0), dim=3, overlap=4.0, wall=1,
                          Vwall_bottom=-0.4, Vwall_top=0.4, dt=2e-5)
    e = sph_b200.System(inp, precision=precision)
    o = oracle.Oracle(inp)
    o.run(0)
    e.step(0)
    o.run(3)
    e.step(3)
    e.synchronize()
    tol = 1e-10 if precision == "fp64" else dict(MIXED_TOL)
    compare_state(e, o, tol, "dense step3")
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), k
    e.close()
    o.close()


@pytest.mark.parametrize("name", list(mg.CASES))
def test_mixed_engine_matches_oracle(name, workdir):
    e, o = open_case(name, workdir, precision="mixed")
    tol = dict(MIXED_TOL)
    tol.update(MIXED_WIDE.get(name, {}))
    o.run(0)
    e.step(0)
    compare_state(e, o, tol, "step0")
    o.run(5)
    e.step(5)
    e.synchronize()
    compare_state(e, o, tol, "step5")


@pytest.mark.parametrize("name", list(mg.CASES))
def test_engine_matches_reference_build(name, workdir):
    """Engine against the reference's own CUDA build (golden dumps)."""
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    e, _ = open_case(name, workdir)
    dim = e.info()["dim"]
    steps = [0] if name == "colloids3d" else mg.steps_of(name)
    done = 0
    for s in steps:
        e.step(s - done)
        e.synchronize()
        done = s
        keys = {k[len("s%d_" % s):] for k in g.files if k.startswith("s%d_" % s)}
        cells = e.export_cells()
        for k in INTS:
            assert np.array_equal(cells[k], g["s%d_%s" % (s, k)]), (s, k)
        for gname, (fields, norm) in GROUPS.items():
            fl = [f for f in fields if f in keys]
            if not fl or gname == "grad":
                continue
            err = group_error(e.field, lambda f: g["s%d_%s" % (s, f)], fl, norm, dim)
            assert err <= (1e-10 if s <= 5 else 1e-9), (s, gname, err)  # 1e-9 after 2000 steps


def test_class_system_methods_step_by_step(workdir):
    """The step methods called one by one, in the order of main.cu:358-467, against the
    oracle after every method (colloids, walls and a body force all active)."""
    e, o = open_case("colloids2d", workdir, use_graph=False)
    tol = 1e-10
    dim = 2

    def check(fields, label, norm="max"):
        err = group_error(e.field, o.field, fields, norm, dim)
        assert err <= tol, (label, err)

    e.neighbours_search()
    o.neighbours_search()
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k))
    for step in range(3):
        t = o.info()["t0"] + o.info()["dt"] * step
        m = o.magnetic_moment(t)
        if step > 0:
            e.V_Verlet_step1()
            o.vv_step1()
            check(["x", "y"], "vv1 pos", "unit")
            check(["vx", "vy"], "vv1 vel")
            e.neighbours_search()
            o.neighbours_search()
            cells = e.export_cells()
            for k in INTS:
                assert np.array_equal(cells[k], o.ifield(k))
        e.calculate_density()
        o.calculate_density()
        check(["dens"], "density")
        e.calculate_pressure()
        o.calculate_pressure()
        check(["press"], "pressure")
        e.calculate_vel_gradient()
        o.calculate_vel_gradient()
        check(["gxx", "gxy", "gyx", "gyy"], "vel_gradient (all particles)")
        e.calculate_forces(m)
        o.calculate_forces(m)
        check(["fx", "fy"], "forces")
        check(["dcdt_xx", "dcdt_xy", "dcdt_yy"], "dcdt")
        for f in ["fx_colloid", "fy_colloid", "tz_colloid"]:
            a, b = e.colloid_field(f), o.field(f)
            assert np.abs(a - b).max() <= tol * np.abs(b).max(), f
        wf = e.wall_forces()[0]
        assert np.abs(wf[:, 0] - o.field("fx_wall")).max() <= tol * np.abs(o.field("fx_wall")).max()
        if step > 0:
            e.V_Verlet_step2()
            o.vv_step2()
            check(["vx", "vy"], "vv2 vel")
            check(["cxx", "cxy", "cyy"], "vv2 conf", "unit")
    ke = e.kinetic_energy()[0]
    assert ke == pytest.approx(o.kinetic_energy(), rel=1e-12)


@pytest.mark.parametrize("name", ["colloids2d", "colloids3d", "couette3d"])
def test_forces_store_the_same_gradient_as_the_gradient_pass(name, workdir):
    """calculate_forces stores the velocity gradient of every particle (walls and colloid
    particles included, kernel_vel_gradients.cu:15-662) from its fused pass: the same bits
    as the standalone calculate_vel_gradient pass, and the same forces after it."""
    mg.case_dir(name, workdir)
    pp = os.path.join(workdir, "input_particles.in")
    pp = [pp] if os.path.exists(pp) else None
    e = sph_b200.System(os.path.join(workdir, "input"), pp, use_graph=False)
    e.step(3)
    grads = ["gxx", "gxy", "gxz", "gyx", "gyy", "gyz", "gzx", "gzy", "gzz"]
    if e.info()["dim"] == 2:
        grads = ["gxx", "gxy", "gyx", "gyy"]
    m = np.array([0.3, 0.4, 0.0])
    e.V_Verlet_step1()
    e.neighbours_search()
    e.calculate_density()
    e.calculate_pressure()
    e.calculate_vel_gradient()
    g_pass = {f: e.field(f) for f in grads}
    e.calculate_forces(m)
    f1 = {f: e.field(f) for f in ["fx", "fy", "fz", "dcdt_xy"]}
    for f in grads:
        assert np.array_equal(e.field(f), g_pass[f]), f
    t = e.type()
    assert (t != 0).sum() > 0
    # the same call again: forces and gradient reproduce
    e.calculate_forces(m)
    for f, v in f1.items():
        assert np.array_equal(e.field(f), v), f
    e.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_neighbour_capacity_grows(precision, workdir):
    """Neighbour lists that start far too short (8 candidate chunks per particle where about
    20 are needed) overflow, are detected on the device, grow and are rebuilt: the run is
    bit-identical to one with the derived capacity, through the step graph and through the
    step methods."""
    mg.case_dir("colloids3d", workdir)
    inp = os.path.join(workdir, "input")
    ref = sph_b200.System(inp, precision=precision)
    small = sph_b200.System(inp, precision=precision, nbr_capacity=8)
    for s in (ref, small):
        s.step(3)
        s.V_Verlet_step1()
        s.neighbours_search()
        s.calculate_forces(np.array([0.2, 0.1, 0.0]))
        s.V_Verlet_step2()
        s.synchronize()
    for f in ["x", "y", "z", "vx", "fx", "dens", "cxy"]:
        assert np.array_equal(small.field(f), ref.field(f)), f
    assert np.array_equal(small.wall_forces(), ref.wall_forces())
    small.close()
    ref.close()


def test_device_errors_are_reported_not_trapped(workdir):
    """A non-finite position and a particle outside the wall band come back as statuses;
    the context keeps working once the state is repaired."""
    e, _ = open_case("couette2d", workdir)
    e.step(1)
    e.synchronize()
    x = e.field("x")
    bad = x.copy()
    bad[10] = np.nan
    e.set_field("x", bad)
    with pytest.raises(sph_b200.SphError) as err:
        e.neighbours_search()
    assert err.value.status == "SPH_ERR_NAN"
    e.set_field("x", x)
    y = e.field("y")
    bad = y.copy()
    bad[5] = -0.5  # far below the bottom wall layers: hashes outside the grid
    e.set_field("y", bad)
    with pytest.raises(sph_b200.SphError) as err:
        e.neighbours_search()
    assert err.value.status == "SPH_ERR_CELL_RANGE"
    e.set_field("y", y)
    e.neighbours_search()
    e.step(2)
    e.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bitwise_reproducible(precision, workdir):
    out = []
    for k in range(2):
        e, _ = open_case("colloids2d", workdir, precision=precision)
        e.step(10)
        e.synchronize()
        out.append(np.concatenate([e.field(f) for f in ["x", "y", "vx", "vy", "fx", "cxy"]] +
                                  [e.colloid_field("coll_x"), e.wall_forces().ravel()]))
        e.close()
    assert np.array_equal(out[0], out[1])


def test_graph_and_direct_paths_agree(workdir):
    a, _ = open_case("couette3d", workdir, use_graph=True)
    b, _ = open_case("couette3d", workdir, use_graph=False)
    a.step(4)
    b.step(4)
    a.synchronize()
    b.synchronize()
    for f in ["x", "vx", "fy", "cxy", "dens"]:
        assert np.array_equal(a.field(f), b.field(f)), f


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["kolmogorov2d", "couette2d", "couette3d"])
def test_step_graph_equals_method_sequence(name, precision, workdir):
    """The step graph, whose pair pass also applies the fluid particles' second half-kick,
    against the class_system call sequence of main.cu:358-467 (V_Verlet_step1,
    neighbours_search, calculate_forces, V_Verlet_step2): the same bits."""
    a, _ = open_case(name, workdir, precision=precision)
    b, _ = open_case(name, workdir, precision=precision)
    a.step(4)
    b.initial_forces()
    for _ in range(4):
        b.V_Verlet_step1()
        b.neighbours_search()
        b.calculate_forces()
        b.V_Verlet_step2()
    a.synchronize()
    b.synchronize()
    fields = ["x", "y", "vx", "vy", "fx", "fy", "dens", "cxx", "cxy", "cyy"]
    if a.info()["dim"] == 3:
        fields += ["z", "vz", "cxz", "cyz", "czz"]
    for f in fields:
        assert np.array_equal(a.field(f), b.field(f)), f
    assert np.array_equal(a.wall_forces(), b.wall_forces())
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_3d_ensemble_equals_single_boxes(precision, workdir):
    """3D boxes in one context against each box alone: a one-box context's pair pass reads
    its constants from the constant bank, an ensemble's from each box's parameters; with
    walls and without, warps clear of the periodic faces and not, the same bits."""
    specs = [
        dict(N=(24, 24, 24), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1, Vwall_top=0.2,
             Vwall_bottom=-0.2, dt=2e-5, tau=0.5),
        dict(N=(20, 16, 18), L=(1.25, 1.0, 1.125), dim=3, overlap=3.0, wall=0, ext_force_type=2,
             ext_force=(1.0, 0.0, 0.0), dt=5e-5),
    ]
    paths = []
    for k, s in enumerate(specs):
        p = os.path.join(workdir, "input%d" % k)
        sph_input.write_input(p, **s)
        paths.append(p)
    ens = sph_b200.System(paths, precision=precision)
    ens.step(5)
    ens.synchronize()
    off = 0
    for k, p in enumerate(paths):
        one = sph_b200.System(p, precision=precision)
        one.step(5)
        one.synchronize()
        n = one.N
        for f in ["x", "y", "z", "vx", "vz", "fx", "fz", "dens", "cxy", "cyz"]:
            assert np.array_equal(ens.field(f)[off:off + n], one.field(f)), (k, f)
        assert np.array_equal(ens.wall_forces()[k], one.wall_forces()[0])
        off += n
        one.close()
    ens.close()


def test_ensemble_equals_single_boxes(workdir):
    """Boxes of different sizes and parameters in one context give, box by box, the same
    bits as each box run alone."""
    specs = [
        dict(N=(32, 32), L=(1.0, 1.0), dim=2, overlap=4.0, wall=1, Vwall_top=0.3,
             Vwall_bottom=-0.3, dt=2e-5, tau=0.5),
        dict(N=(48, 40), L=(1.2, 1.0), dim=2, overlap=4.0, wall=1, Vwall_top=0.1,
             Vwall_bottom=-0.1, dt=2e-5, tau=2.0, N_colloids=2, coll_R=4.0 / 40,
             coll_x=((0.3, 0.5), (0.8, 0.45)), tau_repulsion=5.0, cutoff_magnetic=0.3,
             F0_magnetic=1e-4, F0_repulsion=1e-3, omega_magnetic=3.0),
        dict(N=(40, 40), L=(1.0, 1.0), dim=2, overlap=4.0, wall=0, ext_force_type=2,
             ext_force=(1.0, 0.0), dt=5e-5),
    ]
    paths = []
    for k, s in enumerate(specs):
        p = os.path.join(workdir, "input%d" % k)
        sph_input.write_input(p, **s)
        paths.append(p)
    ens = sph_b200.System(paths)
    ens.step(6)
    ens.synchronize()
    off = 0
    for k, p in enumerate(paths):
        one = sph_b200.System(p)
        one.step(6)
        one.synchronize()
        n = one.N
        for f in ["x", "y", "vx", "vy", "fx", "dens", "cxy"]:
            assert np.array_equal(ens.field(f)[off:off + n], one.field(f)), (k, f)
        assert np.array_equal(ens.wall_forces()[k], one.wall_forces()[0])
        assert ens.kinetic_energy()[k] == one.kinetic_energy()[0]
        off += n
        one.close()


def test_momentum_conserved_periodic(workdir):
    """Pair forces are antisymmetric: without walls, colloids or body force the total
    momentum stays at its initial value to rounding (kernel_forces.cu:429-440)."""
    spec = dict(N=(20, 20, 20), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, dt=2e-5)
    p0 = os.path.join(workdir, "input0")
    sph_input.write_input(p0, **spec)
    o = oracle.Oracle(p0)
    n = o.info()["N"]
    rng = np.random.default_rng(3)
    v = rng.uniform(-0.01, 0.01, size=(3, n))
    pp = os.path.join(workdir, "input_particles.in")
    sph_input.write_particles(pp, 3, o.field("x"), o.field("y"), o.field("z"), v[0], v[1], v[2],
                              o.field("mass"), o.ifield("type"), o.field("cxx"), o.field("cxy"),
                              o.field("cyy"), o.field("cxz"), o.field("cyz"), o.field("czz"))
    path = os.path.join(workdir, "input")
    sph_input.write_input(path, **dict(spec, new_sim=1))
    e = sph_b200.System(path, [pp])
    m = e.field("mass")
    p_init = np.array([np.sum(m * e.field(f)) for f in ["vx", "vy", "vz"]])
    e.step(20)
    e.synchronize()
    p_end = np.array([np.sum(m * e.field(f)) for f in ["vx", "vy", "vz"]])
    scale = np.sum(m * np.abs(e.field("vx")))
    assert np.abs(p_end - p_init).max() <= 1e-12 * scale


def test_full_size_couette_128(workdir):
    """The 128^3 Couette workload (2,195,456 particles): a few steps without errors, the
    lattice neighbourhood of 92 neighbours, FP64 and mixed within the mixed tolerance."""
    spec = dict(N=(128, 128, 128), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0, wall=1,
                Vwall_bottom=-0.5, Vwall_top=0.5, dt=2e-5)
    path = os.path.join(workdir, "input")
    sph_input.write_input(path, **spec)
    a = sph_b200.System(path, precision="fp64")
    assert a.N == 128 * 134 * 128
    a.step(0)
    cells = a.export_cells()
    assert np.all(np.bincount(cells["particle_cell"], minlength=42 * 44 * 42) > 0)
    d = a.field("dens")
    t = a.type()
    assert np.ptp(d[t == 0][:1000]) < 1e-9 * d.mean()
    a.step(3)
    a.synchronize()
    b = sph_b200.System(path, precision="mixed")
    b.step(3)
    b.synchronize()
    for gname in ["pos", "conf", "vel", "dens"]:
        fields, norm = GROUPS[gname]
        err = group_error(b.field, a.field, fields, norm, 3)
        assert err <= MIXED_TOL[gname], (gname, err)
    wa, wb = a.wall_forces(), b.wall_forces()
    assert np.abs(wa - wb).max() <= 2e-5 * np.abs(wa).max()
    # the chunked wall reduction (49,152 particles per wall, 96 chunks) against a host sum
    # of the wall particles' forces (system_calculate_force_walls.cu:15-38)
    t = a.type()
    f = np.stack([a.field("fx"), a.field("fy"), a.field("fz")], axis=1)
    for w in (1, 2):
        ref = f[t == w].sum(axis=0)
        scale = np.abs(f[t == w]).sum(axis=0).max()
        assert np.abs(wa[0, w - 1] - ref).max() <= 1e-12 * scale, (w, wa[0, w - 1], ref)
