"""The CPU oracle against the reference program's own CUDA build.

tests/golden/*.npz hold the state of the reference build (compiled from its unmodified
sources and run on a B200 by tests/golden/make_golden.py) after the initial forces and
after 1 and 5 steps.  The oracle must reproduce every integer array (cell hash, sorted
order, cell ranges, colloid coarse grid) exactly and every real field within 1e-10 of
the field group's scale; the observed differences are at 1e-12 and below and come from
the FMA contractions of nvcc and the CUDA math library.  The 64^2 Kolmogorov case is also
stored after its full 2000 steps, where the bound is 1e-9.

Exception, by design: the reference's 3D colloid velocity-gradient branch writes past a
two-element array (src/kernel_vel_gradients.cu:463-466, 567-570), so its gradients next
to 3D colloids are undefined and differ on the GPU from the intended arithmetic the
oracle follows.  In that case only the step-0 state, which does not yet depend on the
gradient, is compared.
"""
import os

import numpy as np
import pytest

import make_golden as mg
import oracle
from conftest import COLLOID_GROUPS, GROUPS, group_error

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10
# after the 2000 steps of the 64^2 Kolmogorov case the FMA-contraction differences have
# grown to about 1e-10 in the forces (residuals of cancelling pressure terms)
TOL_LONG = 1e-9
INTS = ["type", "particle_cell", "particle_index", "cell_start", "cell_end"]
CINTS = ["coll_cell", "coll_index", "coll_cell_start", "coll_cell_end"]


@pytest.mark.parametrize("name", list(mg.CASES))
def test_oracle_matches_reference_build(name, workdir):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    spec = mg.case_dir(name, workdir)
    pp = os.path.join(workdir, "input_particles.in")
    o = oracle.Oracle(os.path.join(workdir, "input"), pp if os.path.exists(pp) else None)
    dim = o.info()["dim"]
    steps = [0] if name == "colloids3d" else mg.steps_of(name)
    for s in steps:
        o.run(s - o.info()["step"]) if s > 0 else o.run(0)
        keys = {k[len("s%d_" % s):] for k in g.files if k.startswith("s%d_" % s)}
        for k in INTS + CINTS:
            if k in keys:
                assert np.array_equal(o.ifield(k), g["s%d_%s" % (s, k)]), (name, s, k)
        groups = dict(GROUPS)
        if spec.get("N_colloids", 0) if isinstance(spec, dict) else False:
            groups.update(COLLOID_GROUPS)
        for gname, (fields, norm) in groups.items():
            fl = [f for f in fields if f in keys]
            if name == "colloids3d" and gname in ("grad", "dcdt"):
                continue
            if not fl:
                continue
            err = group_error(o.field, lambda f: g["s%d_%s" % (s, f)], fl, norm, dim)
            assert err <= (TOL if s <= 5 else TOL_LONG), (name, s, gname, err)
        if "fx_wall" in keys:
            err = group_error(o.field, lambda f: g["s%d_%s" % (s, f)],
                              ["fx_wall", "fy_wall", "fz_wall"], "max", dim if dim == 3 else 2)
            assert err <= TOL, (name, s, "walls", err)
