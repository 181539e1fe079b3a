"""The allocation-free neighbour search (sph_neighbours_search_noalloc) against the
engine's own search.

The entry point exists for callers that cannot allocate device memory (their memory is
reserved up front by their own allocator, or their time loop must not let an allocation
stall the device); it keeps the sort's scratch in a static device array.  Here it runs
twice in a row on caller-owned arrays (the static scratch keeps the first call's
contents) and must reproduce, bit for bit, the cell arrays the engine exports for the
same positions.  This file is collected last on purpose.
"""
import os

import numpy as np
import pytest

import make_golden as mg
import sph_b200

pytestmark = pytest.mark.gpu


def test_noalloc_search_matches_engine_on_two_calls(tmp_path):
    import torch

    wd = str(tmp_path)
    mg.case_dir("couette3d", wd)
    pp = os.path.join(wd, "input_particles.in")
    e = sph_b200.System(os.path.join(wd, "input"), [pp])
    info = e.info()
    grid = sph_b200.SphGrid(info["dim"], info["wall"], tuple(info["Ncells"]),
                            tuple(info["cell_size"]), info["wall_width"])
    n = e.N
    ncell = info["Ntotal_cells"]
    dev = torch.device("cuda:0")
    pc = torch.empty(n, dtype=torch.int32, device=dev)
    pi = torch.empty(n, dtype=torch.int32, device=dev)
    cs = torch.zeros(ncell, dtype=torch.int32, device=dev)
    ce = torch.zeros(ncell, dtype=torch.int32, device=dev)
    for call in range(2):
        e.step(3)  # moves the particles; the last search of the step saw these positions
        e.synchronize()
        x, y, z = (torch.tensor(e.field(f), dtype=torch.float64, device=dev) for f in "xyz")
        torch.cuda.synchronize()
        st = sph_b200.neighbours_search_noalloc(x.data_ptr(), y.data_ptr(), z.data_ptr(), n,
                                                grid, pc.data_ptr(), pi.data_ptr(),
                                                cs.data_ptr(), ce.data_ptr(), None)
        assert st == 0, sph_b200.STATUS.get(st)
        torch.cuda.synchronize()
        ref = e.export_cells()
        assert np.array_equal(pc.cpu().numpy(), ref["particle_cell"]), call
        assert np.array_equal(pi.cpu().numpy(), ref["particle_index"]), call
        assert np.array_equal(cs.cpu().numpy(), ref["cell_start"]), call
        assert np.array_equal(ce.cpu().numpy(), ref["cell_end"]), call
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
