"""Failures found inside a multi-step (graph-replayed) sph_step call.

A step that finds a problem stops there: its later kernels and every later step of the
call do nothing.  A neighbour list found too short in step k is grown by the next
synchronize, which finishes step k from its list build and runs the remaining steps; the
result must be bit-identical to a run whose lists were long enough throughout.  A bad
position is reported with the step it was found in, and the state is that step's after its
half-kick and drift, the same bits as the class_system method sequence gives.
"""
import os

import numpy as np
import pytest

import make_golden as mg
import sph_b200
import sph_input

pytestmark = pytest.mark.gpu
STATE = ["x", "y", "vx", "vy", "fx", "fy", "dens", "press", "cxx", "cxy", "cyy"]


def converging_box(workdir, A=60.0):
    """64^2 periodic 2D box at overlap 4 (cells of exactly 4 x 4 = 16 particles) whose fluid
    converges on the line y = 0.5 (vy = -A (y - 0.5)): the lattice is compressed along y by
    about A t, so after some 30 steps cells hold a fifth row.  With a half warp per cell
    (candidate chunks of 16 slots) a cell of more than 16 particles gives its neighbours two
    chunks instead of one, and particles need more chunks than at the start."""
    spec = dict(N=(64, 64), L=(1.0, 1.0), dim=2, overlap=4.0, dt=1e-4)
    lat = os.path.join(workdir, "input_lattice")
    sph_input.write_input(lat, **spec)
    a, info = sph_b200.host_setup(lat)
    a = dict(a, vy=-A * (a["y"] - 0.5))
    pp = os.path.join(workdir, "input_particles.in")
    sph_b200.write_restart(pp, 2, a)
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, new_sim=1, **spec)
    return inp, pp


@pytest.mark.parametrize("precision,use_graph", [("fp64", True), ("mixed", True),
                                                 ("fp64", False)])
def test_list_overflow_inside_a_call_resumes(workdir, precision, use_graph):
    inp, pp = converging_box(workdir)
    # the reference run: lists far longer than needed
    ref = sph_b200.System(inp, [pp], precision=precision, use_graph=use_graph, nbr_capacity=64)
    ref.set_tuning(list_threads_per_cell=16)
    ref.step(0)
    need0 = ref.neighbour_lists()["max_used"]
    # lists exactly long enough for the initial search
    tight = sph_b200.System(inp, [pp], precision=precision, use_graph=use_graph,
                            nbr_capacity=need0)
    tight.set_tuning(list_threads_per_cell=16)
    tight.step(0)
    st0 = tight.neighbour_lists()
    assert st0["grown"] == 0 and st0["capacity"] == need0, st0
    nsteps = 50
    ref.step(nsteps)
    tight.step(nsteps)  # one call: the overflow comes in one of its steps
    ref.synchronize()
    tight.synchronize()
    st1 = tight.neighbour_lists()
    assert st1["grown"] >= 1 and st1["max_used"] > st0["capacity"], (st0, st1)
    assert ref.neighbour_lists()["grown"] == 0
    assert tight.info()["step"] == ref.info()["step"] == nsteps
    for f in STATE:
        assert np.array_equal(tight.field(f), ref.field(f)), f
    # and the context goes on
    ref.step(3)
    tight.step(3)
    ref.synchronize()
    tight.synchronize()
    for f in ["x", "vy", "fy", "dens"]:
        assert np.array_equal(tight.field(f), ref.field(f)), f
    ref.close()
    tight.close()


def test_bad_position_stops_the_call_in_its_step(workdir):
    mg.case_dir("colloids2d", workdir)
    inp = os.path.join(workdir, "input")
    a = sph_b200.System(inp)
    b = sph_b200.System(inp)
    for s in (a, b):
        s.step(2)
        s.synchronize()
    vx = a.field("vx")
    vx[7] = np.nan  # the next half-kick and drift give particle 7 a non-finite x
    a.set_field("vx", vx)
    b.set_field("vx", vx)
    a.step(5)
    with pytest.raises(sph_b200.SphError) as err:
        a.synchronize()
    assert err.value.status == "SPH_ERR_NAN"
    assert "in step 3" in str(err.value), str(err.value)
    assert a.info()["step"] == 2
    # the state is step 3's after its half-kick and drift: the method sequence's bits
    b.V_Verlet_step1()
    for f in ["x", "y", "vx", "vy", "cxx", "cxy"]:
        assert np.array_equal(a.field(f), b.field(f), equal_nan=True), f
    assert np.isnan(a.field("x")[7])
    assert np.array_equal(a.colloid_field("coll_x"), b.colloid_field("coll_x"))
    # repaired, the context keeps working
    x = a.field("x")
    x[7] = 0.5
    vx[7] = 0.0
    a.set_field("x", x)
    a.set_field("vx", vx)
    a.neighbours_search()
    a.step(3)
    a.synchronize()
    assert np.all(np.isfinite(a.field("x")))
    a.close()
    b.close()
