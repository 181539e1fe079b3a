"""Known-answer tests of the CPU oracle's kernel functions and neighbour search.

The reference ships no tests or fixtures; these pin the oracle's SPH kernel
(kernel_W.cu:13-59, kernel_gradW.cu:13-53), its cell hash (kernel_cell_list.cu:15-63),
the stable (cell, id) sort order (system_neighbours_search.cu:56-58) and the stale-range
semantics of kernel_cell_ranges.cu:13-33 against closed forms and hand-placed particles.
"""
import math
import os

import numpy as np
import pytest
from scipy.integrate import quad

import oracle
import sph_input


def make(workdir, **kw):
    path = os.path.join(workdir, "input")
    sph_input.write_input(path, **kw)
    return oracle.Oracle(path)


@pytest.mark.parametrize("dim,overlap", [(2, 4.0), (3, 3.0), (2, 3.5)])
def test_kernel_closed_form(workdir, dim, overlap):
    n = (32, 32) if dim == 2 else (24, 24, 24)
    o = make(workdir, N=n, L=(1.0,) * dim, dim=dim, overlap=overlap)
    info = o.info()
    rc, cw = info["rcut"], info["cw"]
    # W(0) = cw (3^5 - 6 * 2^5 + 15) = 66 cw; W and W' vanish at the cutoff
    assert o.W(0.0) == pytest.approx(66.0 * cw, rel=1e-15)
    assert o.W(rc) == 0.0 and o.gradW(rc) == 0.0
    # piecewise quintic in q = 3 r / rcut
    for r in np.linspace(0.0, rc, 41):
        q = 3.0 * r / rc
        w = (3 - q) ** 5 - (6 * (2 - q) ** 5 if q < 2 else 0) + (15 * (1 - q) ** 5 if q < 1 else 0)
        assert o.W(r) == pytest.approx(cw * w, rel=1e-12, abs=1e-12 * cw)
    # the kernel integrates to one
    if dim == 2:
        tot = quad(lambda r: 2 * math.pi * r * o.W(r), 0, rc, points=[rc / 3, 2 * rc / 3])[0]
    else:
        tot = quad(lambda r: 4 * math.pi * r * r * o.W(r), 0, rc, points=[rc / 3, 2 * rc / 3])[0]
    assert tot == pytest.approx(1.0, rel=1e-10)
    # gradW is dW/dr (c_gradw = -15 cw / rcut)
    for r in np.linspace(0.05 * rc, 0.95 * rc, 19):
        h = 1e-7 * rc
        num = (o.W(r + h) - o.W(r - h)) / (2 * h)
        assert o.gradW(r) == pytest.approx(num, rel=1e-6, abs=1e-9 * abs(o.gradW(0.5 * rc)))


def test_cell_hash_sort_and_ranges(workdir):
    # 2D periodic box with 16x16 cells (overlap 4 on a 64^2 lattice)
    o = make(workdir, N=(64, 64), L=(1.0, 1.0), dim=2, overlap=4.0)
    info = o.info()
    n0, n1 = info["Ncells0"], info["Ncells1"]
    cs = info["cell_size0"]
    assert (n0, n1) == (16, 16)
    x, y = o.field("x"), o.field("y")
    # hand-placed particles: x exactly at L hashes to the last cell (clamp), x = 0 to 0
    x[0], y[0] = 1.0, 0.5
    x[1], y[1] = 0.0, 1.0
    x[2], y[2] = 0.999 * cs, 0.0
    o.set_field("x", x)
    o.set_field("y", y)
    assert o.neighbours_search() == 0
    cell, idx = o.ifield("particle_cell"), o.ifield("particle_index")
    expect = {0: 8 * n0 + 15, 1: 15 * n0 + 0, 2: 0}
    inv = np.empty_like(idx)
    inv[idx] = np.arange(idx.size)
    for pid, c in expect.items():
        assert cell[inv[pid]] == c
    # sorted by (cell, id)
    key = cell.astype(np.int64) * idx.size + idx
    assert np.all(np.diff(key) > 0)
    # ranges cover every occupied cell with inclusive ends
    start, end = o.ifield("cell_start"), o.ifield("cell_end")
    occupied = np.unique(cell)
    for c in occupied[:50]:
        members = np.nonzero(cell == c)[0]
        assert start[c] == members[0] and end[c] == members[-1]


def test_stale_ranges_of_emptied_cells(workdir):
    # kernel_cell_ranges.cu writes ranges only for occupied cells; an emptied cell keeps
    # the range of the search that last saw it occupied
    o = make(workdir, N=(64, 64), L=(1.0, 1.0), dim=2, overlap=4.0)
    o.neighbours_search()
    start0, end0 = o.ifield("cell_start").copy(), o.ifield("cell_end").copy()
    x, y = o.field("x"), o.field("y")
    cell = o.ifield("particle_cell")
    idx = o.ifield("particle_index")
    victim = cell[0]  # empty the first cell by moving its particles into cell 5
    cs = o.info()["cell_size0"]
    for k in range(idx.size):
        if cell[k] == victim:
            x[idx[k]] = 5.5 * cs
            y[idx[k]] = 0.5 * cs
    o.set_field("x", x)
    o.set_field("y", y)
    o.neighbours_search()
    assert victim not in set(o.ifield("particle_cell").tolist())
    assert o.ifield("cell_start")[victim] == start0[victim]
    assert o.ifield("cell_end")[victim] == end0[victim]


def test_lattice_density_and_neighbours(workdir):
    # on the initial lattice every particle sees the same neighbourhood: density is uniform
    # and equals the number density 1/dx^d up to the kernel's discretisation error
    o = make(workdir, N=(20, 20, 20), L=(1.0, 1.0, 1.0), dim=3, overlap=3.0)
    o.run(0)
    d = o.field("dens")
    assert np.ptp(d) <= 1e-12 * d.mean()
    assert d.mean() == pytest.approx(20 ** 3, rel=2e-2)
    # fluid at rest on a lattice: no pressure force, no velocity gradient
    assert np.abs(o.field("fx")).max() < 1e-9 * o.field("press").max()
    assert np.abs(o.field("gxy")).max() == 0.0
