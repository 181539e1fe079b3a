"""Observables of an ensemble (sph_observe / sph_observables) against the same quantities
computed from the CPU oracle's state, box by box and step by step."""
import os

import numpy as np
import pytest

import oracle
import sph_b200
import sph_input
from make_golden import CASES

pytestmark = pytest.mark.gpu


def oracle_sample(o, info):
    """One sample: wall shear stress, N1, chain order, kinetic energy (as sph_capi.h)."""
    dim = info["dim"]
    L = [info["L0"], info["L1"], info["L2"]]
    tw = -o.field("fx_wall")[1] / (L[0] * (L[2] if dim == 3 else 1.0)) if info["wall"] else 0.0
    t = o.ifield("type")
    fl = t == 0
    n1 = float(np.mean(info["nkT"] * (o.field("cxx")[fl] - o.field("cyy")[fl])))
    chain = 0.0
    n = info["N_colloids"]
    if n >= 2:
        step = info["step"]
        ang = info["omega_magnet"] * (info["t0"] + info["dt"] * step)
        m = np.array([np.cos(ang), np.sin(ang), 0.0])
        xs = np.stack([o.field("coll_x"), o.field("coll_y"),
                       o.field("coll_z") if dim == 3 else np.zeros(n)], axis=1)
        vals = []
        for a in range(n):
            for b in range(a + 1, n):
                r = xs[a] - xs[b]
                for k in range(3 if dim == 3 else 2):
                    if k == 1 and info["wall"]:
                        continue
                    if r[k] > 0.5 * L[k]:
                        r[k] -= L[k]
                    if r[k] < -0.5 * L[k]:
                        r[k] += L[k]
                r2 = float(r @ r)
                if 0 < r2 < (2.5 * info["coll_R"]) ** 2:
                    c = float(r @ m) / (np.sqrt(r2) * np.linalg.norm(m))
                    vals.append(1.5 * c * c - 0.5 if dim == 3 else 2 * c * c - 1)
        chain = float(np.mean(vals)) if vals else 0.0
    return np.array([tw, n1, chain, o.kinetic_energy()])


def test_observables_match_oracle(workdir):
    specs = [CASES["colloids2d"], CASES["couette2d"]]
    paths = []
    for k, s in enumerate(specs):
        p = os.path.join(workdir, "input%d" % k)
        sph_input.write_input(p, **s)
        paths.append(p)
    ens = sph_b200.System(paths)
    nsteps = 6
    for _ in range(nsteps):
        ens.step(1)
        ens.observe()
    avg, nsamp = ens.observables()
    assert nsamp == nsteps
    for b, p in enumerate(paths):
        o = oracle.Oracle(p)
        acc = np.zeros(4)
        for s in range(nsteps):
            o.run(1)
            acc += oracle_sample(o, o.info())
        want = acc / nsteps
        scale = np.maximum(np.abs(want), 1e-300)
        err = np.abs(avg[b] - want) / scale
        assert np.all((err <= 1e-9) | (np.abs(avg[b] - want) <= 1e-14)), (b, avg[b], want)
        o.close()
    # the 2D colloid box has a bond within 2.5 R, so the chain order is a real sample
    assert avg[0, 2] != 0.0
    ens.reset_observables()
    avg, nsamp = ens.observables()
    assert nsamp == 0 and np.all(avg == 0)
    ens.close()
