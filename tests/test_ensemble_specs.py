"""The batched workload's boxes (sph_ensemble): every sampled sweep point builds through
the engine's host set-up (the reference's own input checks), within the stated ranges and
feasibility rules.  Host code only."""
import math

import numpy as np

import sph_b200
import sph_ensemble
import sph_input


def test_all_512_boxes_are_valid(tmp_path):
    pts = sph_ensemble.draw_points(512, seed=0)
    paths, specs = sph_ensemble.write_inputs(pts, str(tmp_path), nsteps=100)
    sizes = []
    for pt, spec, p in zip(pts, specs, paths):
        assert 32 <= pt["N"] <= 128
        assert 0.1 <= pt["tau"] <= 10 and 0.1 <= pt["omega_tau"] <= 10
        assert 0.1 <= pt["F0_ratio"] <= 2 and 0.1 <= pt["Vwall"] <= 1 and 0.5 <= pt["nkT"] <= 2
        assert spec["N_colloids"] <= pt["ncoll"] <= 24
        R = spec["coll_R"]
        c = np.array(spec["coll_x"]).reshape(-1, 2)
        for a in range(len(c)):
            for b in range(a + 1, len(c)):
                dx = c[a, 0] - c[b, 0]
                dx -= round(dx)
                assert math.hypot(dx, c[a, 1] - c[b, 1]) >= 2.2 * R - 1e-12
        st = sph_b200.host_setup(p)  # raises on any input the reference would reject
        info = [x for x in st if isinstance(x, dict) and "N" in x][0]
        if spec["N_colloids"] > 0:
            assert min(info["Ncells_colloids"][:2]) >= 3
        sizes.append(info["N"])
    # uneven sizes, about 4 million particles in all
    assert min(sizes) < 1500 and max(sizes) > 15000
    assert 3e6 < sum(sizes) < 6e6
    # points with colloids exist across the size range
    assert sum(1 for s in specs if s["N_colloids"] > 0) > 400


def test_features_are_the_six_inputs():
    pt = sph_ensemble.draw_points(1, seed=5)[0]
    spec = sph_ensemble.box_spec(pt)
    f = sph_ensemble.features(pt, spec)
    assert f.shape == (len(sph_ensemble.FEATURES),)
    assert f[0] == 2 * pt["Vwall"] * pt["tau"]
    assert f[2] == spec["N_colloids"] * math.pi * spec["coll_R"] ** 2
    text = sph_input.make_input(**spec)
    assert "omega_magnetic" in text and "coll_x" in text
