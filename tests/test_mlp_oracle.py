"""The FP64 network oracle (oracle/mlp_oracle.py) itself: its analytic gradient against
finite differences, and bf16 rounding to nearest-even.  CPU only."""
import numpy as np

import mlp_oracle


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.1, mlp_oracle.NPARAMS)
    x = rng.normal(size=(16, 6))
    y = rng.normal(size=(16, 4))
    loss, g = mlp_oracle.loss_and_grads(p, x, y, bf16_like_gpu=False)
    for name in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        a, b = mlp_oracle.OFFS[name]
        for i in rng.integers(a, b, 3):
            e = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[i] += e
            pm[i] -= e
            fd = (mlp_oracle.loss_and_grads(pp, x, y, False)[0] -
                  mlp_oracle.loss_and_grads(pm, x, y, False)[0]) / (2 * e)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (name, i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 1e-3])
    r = mlp_oracle.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0            # tie, to even
    assert r[2] == 1.0 + 2 ** -7  # tie, to even (up)
    assert r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 1e-3) <= 2 ** -9 * 1e-3
