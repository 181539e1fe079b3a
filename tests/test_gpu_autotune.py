"""Launch geometry (sph_set_tuning) and the autotuner (sph_autotune): every geometry gives
the same bits, autotuning leaves the simulation state unchanged, and the cache file is
written once and then reused."""
import json
import os

import numpy as np
import pytest

import sph_b200
import sph_input
from make_golden import CASES

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "vx", "vy", "fx", "fy", "dens", "cxy"]


def _input(workdir, name, **over):
    p = os.path.join(workdir, "input_" + name)
    sph_input.write_input(p, **dict(CASES[name], **over))
    return p


@pytest.mark.parametrize("case", ["colloids2d", "couette2d", "kolmogorov2d"])
def test_geometries_give_identical_bits(workdir, case):
    p = _input(workdir, case)
    runs = []
    for tpc, blk in [(32, 128), (16, 64), (16, 256), (32, 256), (32, 0), (16, 0)]:
        s = sph_b200.System(p)
        s.set_tuning(tpc, blk)
        assert s.tuning() == {"list_threads_per_cell": tpc, "density_block": blk}
        s.step(6)
        s.synchronize()
        runs.append({f: s.field(f) for f in FIELDS} | {"cells": s.export_cells()["cell_start"]})
        s.close()
    for r in runs[1:]:
        for f in FIELDS:
            assert np.array_equal(r[f], runs[0][f]), f


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_3d_density_tiles_identical(workdir, precision):
    """The density pass over neighbour-cell tiles against the per-particle pass, in 3D with
    colloids (stale and empty cells inside them) and at overlap 4, where 9 cells of 64
    particles overflow the tile and the overflow is read from global memory."""
    p3 = _input(workdir, "colloids3d")
    p4 = os.path.join(workdir, "input_ov4")
    sph_input.write_input(p4, N=(24, 24, 24), L=(1.0, 1.0, 1.0), dim=3, overlap=4.0, wall=1,
                          Vwall_bottom=-0.3, Vwall_top=0.3, dt=2e-5)
    for p in (p3, p4):
        out = []
        for blk in (128, 0):
            s = sph_b200.System(p, precision=precision)
            s.set_tuning(32, blk)
            s.step(3)
            s.synchronize()
            out.append([s.field(f) for f in ("x", "vx", "fz", "dens", "press")])
            s.close()
        for a, b in zip(*out):
            assert np.array_equal(a, b)


def test_3d_half_warp_lists_identical(workdir):
    p = _input(workdir, "colloids3d")
    out = []
    for tpc in (32, 16):
        s = sph_b200.System(p)
        s.set_tuning(tpc, 128)
        s.step(3)
        s.synchronize()
        out.append([s.field(f) for f in ("x", "vx", "fz", "dens")])
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_autotune_keeps_state_and_caches(workdir):
    p = _input(workdir, "colloids2d")
    cache = os.path.join(workdir, "tune.json")
    plain = sph_b200.System(p)
    plain.step(2)
    plain.synchronize()
    tuned = sph_b200.System(p)
    tuned.step(2)
    tuned.synchronize()
    choice = tuned.autotune(cache)
    assert choice["list_threads_per_cell"] in (16, 32)
    assert choice["density_block"] in (0, 64, 128, 256)  # 0: the neighbour-cell tile pass
    assert tuned.tuning() == choice
    for s in (plain, tuned):
        s.step(4)
        s.synchronize()
    for f in FIELDS:
        assert np.array_equal(plain.field(f), tuned.field(f)), f
    entries = json.load(open(cache))
    assert len(entries) == 1
    key, val = next(iter(entries.items()))
    assert "|dim=2|" in key and val["list_threads_per_cell"] == choice["list_threads_per_cell"]
    # a second context of the same kind takes the cached choice
    before = open(cache).read()
    other = sph_b200.System(p)
    assert other.autotune(cache) == choice
    assert open(cache).read() == before
    # a different kind of box adds its own entry
    q = _input(workdir, "kolmogorov2d")
    third = sph_b200.System(q)
    third.autotune(cache)
    assert len(json.load(open(cache))) == 2
    for s in (plain, tuned, other, third):
        s.close()


def test_bad_geometry_rejected(workdir):
    s = sph_b200.System(_input(workdir, "couette2d"))
    with pytest.raises(sph_b200.SphError):
        s.set_tuning(8, 128)
    with pytest.raises(sph_b200.SphError):
        s.set_tuning(32, 96)
    s.close()
