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
