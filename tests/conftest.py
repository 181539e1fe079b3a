import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sph-magnetic-particles-oldroyd-b-in-cuda_b200")
for p in (os.path.join(ROOT, "oracle"), PKG, os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the engine)")


# Field groups and how their errors are normalised: positions by the box (L = 1) and the
# conformation tensor by its natural scale 1; every other group by the largest magnitude
# of the reference values in that group.
GROUPS = {
    "pos": (["x", "y", "z"], "unit"),
    "vel": (["vx", "vy", "vz"], "max"),
    "force": (["fx", "fy", "fz"], "max"),
    "dens": (["dens"], "max"),
    "press": (["press"], "max"),
    "conf": (["cxx", "cxy", "cyy", "cxz", "cyz", "czz"], "unit"),
    "dcdt": (["dcdt_xx", "dcdt_xy", "dcdt_yy", "dcdt_xz", "dcdt_yz", "dcdt_zz"], "max"),
    "grad": (["gxx", "gxy", "gxz", "gyx", "gyy", "gyz", "gzx", "gzy", "gzz"], "max"),
}
COLLOID_GROUPS = {
    "cpos": (["coll_x", "coll_y", "coll_z"], "unit"),
    "cvel": (["coll_vx", "coll_vy", "coll_vz"], "max"),
    "comega": (["coll_omegax", "coll_omegay", "coll_omegaz"], "max"),
    "cforce": (["fx_colloid", "fy_colloid", "fz_colloid"], "max"),
    "ctorque": (["tx_colloid", "ty_colloid", "tz_colloid"], "max"),
}
TWO_D_ONLY = {"z", "vz", "fz", "cxz", "cyz", "czz", "dcdt_xz", "dcdt_yz", "dcdt_zz", "gxz",
              "gyz", "gzx", "gzy", "gzz", "coll_z", "coll_vz", "coll_omegax", "coll_omegay",
              "fz_colloid", "tx_colloid", "ty_colloid"}


def group_error(get_a, get_b, fields, norm, dim):
    """max |a - b| over the group, divided by the group's scale."""
    fl = [f for f in fields if dim == 3 or f not in TWO_D_ONLY]
    a = np.concatenate([np.asarray(get_a(f), dtype=np.float64) for f in fl])
    b = np.concatenate([np.asarray(get_b(f), dtype=np.float64) for f in fl])
    if a.size == 0:
        return 0.0
    scale = 1.0 if norm == "unit" else float(np.abs(b).max())
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))


@pytest.fixture
def workdir(tmp_path):
    return str(tmp_path)
