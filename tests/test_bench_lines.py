"""bench.py's JSON line builders run on the CPU with stand-in numbers, so that a GPU run
never fails at its last line."""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_sweep_line_is_json():
    args = argparse.Namespace(precision="mixed", sweep_train_steps=3000)
    rng = np.random.default_rng(0)
    Yte = rng.normal(1, 0.3, (512, 4))
    line = bench.sweep_line(args, 2000, 20480, 65536, [0.5, 0.6], 300.0, 20992, 5.0, 0.1, 40.0,
                            Yte * 1.001, rng.random(512) < 0.1, Yte, Yte, rng.random(65536) < 0.1)
    text = json.dumps(line)
    assert json.loads(text)["unit"] == "points/h"
    assert line["value"] > 0 and line["accepted"] is True
    assert "2000 steps" in line["config"]["workload"]


def test_single_box_workloads_write_their_inputs(tmp_path):
    """The couette3d workload writes the seeded restart start beside its input; the
    suspension96 workload writes the lattice input of config 3 with the scaled amplitudes."""
    import bench

    (tmp_path / "c").mkdir()
    (tmp_path / "s").mkdir()
    c = bench.WORKLOADS["couette3d"]
    inp = c.write(str(tmp_path / "c"), lattice=12)
    assert bench.particles_file(inp) is not None and "new_sim 1" in open(inp).read()
    s = bench.WORKLOADS["suspension96"]
    inp = s.write(str(tmp_path / "s"), lattice=96)
    text = open(inp).read()
    assert bench.particles_file(inp) is None
    assert text.count("coll_x ") == 32 and "F0_magnetic 0.0005" in text
