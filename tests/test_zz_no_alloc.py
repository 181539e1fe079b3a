"""The allocation-free neighbour search (sph_neighbours_search_noalloc) against the
engine's own search.

The entry point exists for callers that cannot allocate device memory: programs whose
device memory is reserved up front by their own allocator, where a cudaMalloc would fail
or take memory the allocator counts on, and time loops that must not let an allocation
(which can synchronise the whole device) stall them.  It keeps the sort's scratch in a
static device array.  Here it runs twice in a row on caller-owned arrays (the static
scratch keeps the first call's contents) and must reproduce, bit for bit, the cell arrays
the engine exports for the same positions, while the device's free memory stays exactly
the same across each call.  This file is collected last on purpose.
"""
import os

import numpy as np
import pytest

import make_golden as mg
import sph_b200

pytestmark = pytest.mark.gpu
INTS = ["particle_cell", "particle_index", "cell_start", "cell_end"]


def _grid(e):
    info = e.info()
    return sph_b200.SphGrid(info["dim"], info["wall"], tuple(info["Ncells"]),
                            tuple(info["cell_size"]), info["wall_width"]), info


class Buffers:
    """Caller-owned device arrays, allocated once (torch) before anything is measured."""

    def __init__(self, n, ncell, dim):
        import torch

        dev = torch.device("cuda:0")
        self.torch = torch
        self.dim = dim
        self.pos = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(dim)]
        self.pc = torch.empty(n, dtype=torch.int32, device=dev)
        self.pi = torch.empty(n, dtype=torch.int32, device=dev)
        self.cs = torch.zeros(ncell, dtype=torch.int32, device=dev)
        self.ce = torch.zeros(ncell, dtype=torch.int32, device=dev)

    def load(self, arrays):
        for dst, src in zip(self.pos, arrays):
            dst.copy_(self.torch.from_numpy(np.ascontiguousarray(src, dtype=np.float64)))
        self.torch.cuda.synchronize()

    def call(self, grid, n):
        z = self.pos[2].data_ptr() if self.dim == 3 else None
        return sph_b200.neighbours_search_noalloc(self.pos[0].data_ptr(), self.pos[1].data_ptr(),
                                                  z, n, grid, self.pc.data_ptr(),
                                                  self.pi.data_ptr(), self.cs.data_ptr(),
                                                  self.ce.data_ptr(), None)

    def measured_call(self, grid, n):
        """One call with the device's free memory read before and after it."""
        torch = self.torch
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st = self.call(grid, n)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert free1 == free0, ("device memory changed during the call", free0, free1)
        return st

    def result(self):
        return {"particle_cell": self.pc.cpu().numpy(), "particle_index": self.pi.cpu().numpy(),
                "cell_start": self.cs.cpu().numpy(), "cell_end": self.ce.cpu().numpy()}


def _positions(e, dim):
    return [e.field(f) for f in ("x", "y", "z")[:dim]]


def _assert_cells_equal(got, ref, label):
    for k in INTS:
        assert np.array_equal(got[k], ref[k]), (label, k)


def _warm(buf, grid, e, dim):
    """A first call with one particle: the driver places this entry point's device code and
    its static scratch array when they are first used; calls after that allocate nothing."""
    buf.load(_positions(e, dim))
    assert buf.call(grid, 1) == 0


def _two_calls(name, workdir, steps=3):
    mg.case_dir(name, workdir)
    pp = os.path.join(workdir, "input_particles.in")
    e = sph_b200.System(os.path.join(workdir, "input"), [pp] if os.path.exists(pp) else None)
    grid, info = _grid(e)
    dim, n = info["dim"], e.N
    buf = Buffers(n, info["Ntotal_cells"], dim)
    e.step(1)
    e.synchronize()
    _warm(buf, grid, e, dim)
    for call in range(2):
        e.step(steps)  # moves the particles; the last search of the step saw these positions
        e.synchronize()
        buf.load(_positions(e, dim))
        st = buf.measured_call(grid, n)
        assert st == 0, sph_b200.STATUS.get(st)
        _assert_cells_equal(buf.result(), e.export_cells(), (name, call))
    e.close()
    return info


def test_noalloc_search_matches_engine_on_two_calls(workdir):
    """3D walls box (16^3 from seeded velocities), z passed."""
    _two_calls("couette3d", workdir)


def test_noalloc_search_2d_without_z(workdir):
    """2D box: z is NULL, as a 2D caller passes it."""
    info = _two_calls("couette2d", workdir)
    assert info["dim"] == 2


def test_noalloc_search_two_sort_passes(workdir):
    """32^3 periodic box with colloids: 1,000 cells need 10 key bits, sorted in two passes."""
    info = _two_calls("colloids3d", workdir, steps=2)
    assert info["Ntotal_cells"] > 512


@pytest.mark.parametrize("bad", ["outside", "nan"])
def test_noalloc_status_is_cleared_between_calls(workdir, bad):
    """A position outside the grid (or not a number) gives SPH_ERR_CELL_RANGE; the next call
    on valid positions succeeds and matches the engine, so the status word was cleared."""
    mg.case_dir("couette2d", workdir)
    e = sph_b200.System(os.path.join(workdir, "input"))
    grid, info = _grid(e)
    n = e.N
    buf = Buffers(n, info["Ntotal_cells"], 2)
    e.step(1)
    e.synchronize()
    _warm(buf, grid, e, 2)
    x, y = _positions(e, 2)
    xb, yb = x.copy(), y.copy()
    if bad == "outside":
        yb[n // 3] = 50.0  # a cell row far above the grid: linear cell index past the end
    else:
        xb[n // 3] = np.nan
    buf.load([xb, yb])
    st = buf.measured_call(grid, n)
    assert sph_b200.STATUS[st] == "SPH_ERR_CELL_RANGE"
    buf.load([x, y])
    st = buf.measured_call(grid, n)
    assert st == 0, sph_b200.STATUS.get(st)
    _assert_cells_equal(buf.result(), e.export_cells(), "clean call after " + bad)
    e.close()


def test_noalloc_rejects_more_than_its_maximum():
    grid = sph_b200.SphGrid(3, 0, (4, 4, 4), (0.25, 0.25, 0.25), 0.0)
    too_many = (1 << 20) + 1
    st = sph_b200.neighbours_search_noalloc(None, None, None, too_many, grid, None, None, None,
                                            None, None)
    assert sph_b200.STATUS[st] == "SPH_ERR_BAD_INPUT"  # null arrays are refused first
    import torch

    buf = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    ibuf = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    p, q = buf.data_ptr(), ibuf.data_ptr()
    st = sph_b200.neighbours_search_noalloc(p, p, p, too_many, grid, q, q, q, q, None)
    assert sph_b200.STATUS[st] == "SPH_ERR_CAPACITY"
