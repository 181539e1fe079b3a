"""The benchmark workload itself at full size: 128^3 Oldroyd-B Couette flow between y-walls
(2,195,456 particles) from the seeded start the benchmark runs (bench.write_workload: fluid
velocities uniform in +-1e-3 c, read by every implementation through new_sim = 1 and the
restart file), FP64 engine against the FP64 oracle after the initial forces, 1 step and
5 steps.

Tolerance: every field group within 1e-10 of its scale (conftest.GROUPS), the wall forces
within 1e-10 of their largest component; the exported cell / sort arrays
(particle_cell, particle_index, cell_start, cell_end) bit-exact.  The oracle is built
without FMA contraction, the engine with it, so the two differ by rounding only.
"""
import os
import sys

import numpy as np
import pytest

import oracle
import sph_b200
from conftest import GROUPS, group_error

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402

pytestmark = pytest.mark.gpu
INTS = ["particle_cell", "particle_index", "cell_start", "cell_end"]


def compare(e, o, label):
    errs = {}
    for gname, (fields, norm) in GROUPS.items():
        if gname == "grad":
            continue
        errs[gname] = group_error(e.field, o.field, fields, norm, 3)
    wf = e.wall_forces()[0]
    ref = np.stack([o.field("fx_wall"), o.field("fy_wall"), o.field("fz_wall")], axis=1)
    errs["walls"] = float(np.abs(wf - ref).max() / np.abs(ref).max())
    for k, v in errs.items():
        assert v <= 1e-10, (label, k, v)
    cells = e.export_cells()
    for k in INTS:
        assert np.array_equal(cells[k], o.ifield(k)), (label, k)
    return errs


def test_couette128_seeded_fp64_matches_oracle(workdir):
    inp = bench.write_workload(workdir)
    pp = bench.particles_file(inp)
    oracle.set_threads(os.cpu_count() or 1)
    e = sph_b200.System(inp, [pp], precision="fp64")
    o = oracle.Oracle(inp, pp)
    assert e.N == o.info()["N"] == 128 * 134 * 128
    v = e.field("vx")
    fluid = e.type() == 0
    assert 0.004 < np.std(v[fluid]) and np.abs(v).max() <= bench.VMAX  # the seeded start
    o.run(0)
    e.step(0)
    compare(e, o, "step0")
    o.run(1)
    e.step(1)
    e.synchronize()
    compare(e, o, "step1")
    o.run(4)
    e.step(4)
    e.synchronize()
    errs = compare(e, o, "step5")
    assert e.info()["step"] == o.info()["step"] == 5, errs
    e.close()
    o.close()
