"""What the trained network gains over the method without it, on a small sweep: the
surrogate, trained on the batched solver's output, predicts held-out points (re-solved by
the solver) far better than the best constant predictor, and its heads flag the points
it is unsure of."""
import numpy as np
import pytest

import sph_ensemble
import sph_surrogate

pytestmark = pytest.mark.gpu


def test_surrogate_beats_constant_predictor_on_heldout_points():
    nsteps, ntrain = 400, 1024
    pts = sph_ensemble.draw_points(ntrain + 256, seed=4, fixed_N=32, coll_seed=3)
    Y, secs = sph_surrogate.solve_points(pts, nsteps, "mixed")
    assert np.all(np.isfinite(Y))
    X = sph_surrogate.features_of(pts)
    Xtr, Ytr, Xte, Yte = X[:ntrain], Y[:ntrain], X[ntrain:], Y[ntrain:]
    sur = sph_surrogate.Surrogate(heads=5, seed=1)
    sur.fit(Xtr, Ytr, steps=1500)
    mean, route = sur.predict(Xte)
    # wall shear stress (the routed target) and the kinetic energy
    for k in (0, 3):
        err = sph_surrogate.relative_error(mean[:, k], Yte[:, k])
        const = sph_surrogate.relative_error(np.full(len(Yte), Ytr[:, k].mean()), Yte[:, k])
        assert err < 0.1 * const, (k, err, const)
    # points the heads agree on are predicted at least as well as the rest
    keep = ~route
    assert keep.sum() > len(keep) // 2
    e_keep = sph_surrogate.relative_error(mean[keep, 0], Yte[keep, 0])
    assert e_keep <= sph_surrogate.relative_error(mean[:, 0], Yte[:, 0]) * 1.05
    sur.mlp.close()
