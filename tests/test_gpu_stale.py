"""Stale cell ranges and positions outside the box, engine against the FP64 oracle.

kernel_cell_ranges.cu:13-33 writes cell_start / cell_end only for occupied cells, so a
cell emptied since an earlier search keeps its old range.  After the sort those slots hold
other particles, and the density and force loops (kernel_densities.cu:52-163,
kernel_forces.cu) take them by the minimum image like any candidate: a particle next to
the emptied cell sums some neighbours twice.  Emptying the last cell of a row puts the
first particles of the next row, across the periodic x face, in the stale slots; the
engine must list them at their minimum image, not with the emptied cell's (zero) shift.

A position outside [0, L] that the cell hash still accepts (x = L + 1.5 cells is
clamped into the next row, kernel_cell_list.cu:15-63) makes a particle clear of the
periodic faces see a neighbour only through the minimum image: the pair passes must keep
it for every particle then.

Tolerances: densities within 1e-12 and forces, dc/dt within 1e-10 of their scales; cell
arrays bit-exact.
"""
import os

import numpy as np
import pytest

import oracle
import sph_b200
import sph_input

pytestmark = pytest.mark.gpu
INTS = ["particle_cell", "particle_index", "cell_start", "cell_end"]


def pair(workdir, tpc, **kw):
    inp = os.path.join(workdir, "input")
    sph_input.write_input(inp, **kw)
    e = sph_b200.System(inp, precision="fp64")
    e.set_tuning(list_threads_per_cell=tpc, density_block=128)
    return e, oracle.Oracle(inp)


def both(e, o, name, *args):
    getattr(e, name)(*args)
    getattr(o, name if name != "V_Verlet_step1" else "vv_step1")(*args)


def check(e, o, fields, tol, label):
    for f in fields:
        a, b = e.field(f), o.field(f)
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
        assert err <= tol, (label, f, err)


def check_cells(e, o):
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), k


def brute_density(o, dim):
    """Density without the stale double counts: every pair within rcut once (unit box)."""
    x = np.stack([o.field(c) for c in ("x", "y", "z")[:dim]], 1)
    rc = o.info()["rcut"]
    out = np.empty(len(x))
    for i in range(len(x)):
        r = x - x[i]
        r -= np.round(r)
        rr = np.sqrt((r * r).sum(1))
        out[i] = sum(o.W(v) for v in rr[rr < rc])
    return out


def move_cell(o, e, cell_id, target, dim):
    """Moves every particle of cell `cell_id` onto a small grid (spacing 0.21 cells, off
    the lattice) from `target`, a point inside the box."""
    cell, idx = o.ifield("particle_cell"), o.ifield("particle_index")
    cs = o.info()["cell_size0"]
    pos = {c: o.field(c) for c in ("x", "y", "z")[:dim]}
    moved = [int(idx[k]) for k in range(idx.size) if cell[k] == cell_id]
    assert moved
    side = 4 if dim == 2 else 3
    for n, pid in enumerate(moved):
        for a, c in enumerate(("x", "y", "z")[:dim]):
            pos[c][pid] = target[a] + 0.21 * cs * ((n // side ** a) % side)
    for c, v in pos.items():
        o.set_field(c, v)
        e.set_field(c, v)


@pytest.mark.parametrize("tpc", [32, 16])
def test_stale_range_across_the_x_face_2d(workdir, tpc):
    e, o = pair(workdir, tpc, N=(64, 64), L=(1.0, 1.0), dim=2, overlap=4.0)
    both(e, o, "neighbours_search")
    n0, cs = o.info()["Ncells0"], o.info()["cell_size0"]
    victim = 5 * n0 + (n0 - 1)  # the last cell of row 5
    start0 = o.ifield("cell_start")[victim]
    move_cell(o, e, victim, (5.5 * cs, 9.5 * cs), 2)
    both(e, o, "neighbours_search")
    check_cells(e, o)
    assert o.ifield("cell_start")[victim] == start0  # stale
    both(e, o, "calculate_density")
    check(e, o, ["dens"], 1e-12, "density")
    # the oracle's sums hold the reference's double counts next to the emptied cell
    bd = brute_density(o, 2)
    assert np.abs(o.field("dens") - bd).max() > 1e-6 * bd.max()
    both(e, o, "calculate_pressure")
    both(e, o, "calculate_forces", np.zeros(3))
    check(e, o, ["fx", "fy", "dcdt_xx", "dcdt_xy", "dcdt_yy"], 1e-10, "forces")


@pytest.mark.parametrize("tpc", [32, 16])
def test_stale_range_across_the_x_face_3d(workdir, tpc):
    e, o = pair(workdir, tpc, N=(24, 24, 24), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0)
    both(e, o, "neighbours_search")
    n0, n1 = o.info()["Ncells0"], o.info()["Ncells1"]
    cs = o.info()["cell_size0"]
    victim = (3 * n1 + 4) * n0 + (n0 - 1)  # the last cell of row (y 4, z 3)
    move_cell(o, e, victim, (3.5 * cs, 1.5 * cs, 6.5 * cs), 3)
    both(e, o, "neighbours_search")
    check_cells(e, o)
    both(e, o, "calculate_density")
    check(e, o, ["dens"], 1e-12, "density")
    bd = brute_density(o, 3)
    assert np.abs(o.field("dens") - bd).max() > 1e-6 * bd.max()
    both(e, o, "calculate_pressure")
    both(e, o, "calculate_forces", np.zeros(3))
    check(e, o, ["fx", "fy", "fz", "dcdt_xx", "dcdt_xy", "dcdt_yy", "dcdt_xz", "dcdt_yz",
                 "dcdt_zz"], 1e-10, "forces")


def test_position_outside_the_box_keeps_the_minimum_image(workdir):
    # 64^2 lattice, 16 x 16 cells of 4 spacings (= rcut)
    e, o = pair(workdir, 32, N=(64, 64), L=(1.0, 1.0), dim=2, overlap=4.0)
    both(e, o, "neighbours_search")
    dx = 1.0 / 64
    x, y = o.field("x"), o.field("y")
    # i: a lattice particle 8.5 spacings from the x face (clear of it), row of cells 6
    i = int(np.argmin((x - 8.5 * dx) ** 2 + (y - 24.5 * dx) ** 2))
    assert abs(x[i] - 8.5 * dx) < 1e-12
    # j: x = L + 6 spacings hashes to cell x 1 of the next row; its image is 2.5 spacings
    # from i, within the cutoff only through the minimum image
    j = int(np.argmin((x - 40.5 * dx) ** 2 + (y - 40.5 * dx) ** 2))
    x[j], y[j] = 1.0 + 6.0 * dx, y[i] - 0.1 * dx
    for name, v in (("x", x), ("y", y)):
        o.set_field(name, v)
        e.set_field(name, v)
    both(e, o, "neighbours_search")
    check_cells(e, o)
    both(e, o, "calculate_density")
    check(e, o, ["dens"], 1e-12, "density")
    both(e, o, "calculate_pressure")
    both(e, o, "calculate_forces", np.zeros(3))
    check(e, o, ["fx", "fy", "dcdt_xx", "dcdt_xy", "dcdt_yy"], 1e-10, "forces")
    # the pair (i, j) is in the sums: i's density exceeds a lattice particle's
    d = o.field("dens")
    assert d[i] > np.median(d) * (1 + 1e-6)
