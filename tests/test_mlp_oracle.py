"""The FP64 numpy MLP (oracle/mlp_oracle.py) and the normalisation folding of
warpvbd_b200.warmstart, on the CPU."""
import numpy as np

from oracle import mlp_oracle as mo
from warpvbd_b200 import warmstart as ws


def test_layout_matches_library_constants():
    assert mo.N_PARAMS == ws.N_PARAMS == 5827


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(3)
    p = ws.init_params(1).astype(np.float64) + rng.normal(scale=0.05, size=mo.N_PARAMS)
    X = rng.normal(size=(7, 24))
    Y = rng.normal(size=(7, 3))
    _, g, _ = mo.loss_and_grad(p, X, Y)
    for i in rng.choice(mo.N_PARAMS, size=60, replace=False):
        e = np.zeros(mo.N_PARAMS)
        e[i] = 1e-6
        lp, _, _ = mo.loss_and_grad(p + e, X, Y)
        lm, _, _ = mo.loss_and_grad(p - e, X, Y)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) < 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_fold_normalization_is_exact():
    rng = np.random.default_rng(4)
    p = ws.init_params(2)
    X = rng.normal(loc=3.0, scale=2.0, size=(50, 24))
    mu_x, sd_x = X[:, :22].mean(0), X[:, :22].std(0)
    mu_y, sd_y = rng.normal(size=3), rng.uniform(0.5, 2.0, size=3)
    Xn = X.copy()
    Xn[:, :22] = (X[:, :22] - mu_x) / sd_x
    out_n, _ = mo.forward(p.astype(np.float64), Xn)
    raw = ws.fold_normalization(p, mu_x, sd_x, mu_y, sd_y)
    out_raw, _ = mo.forward(raw.astype(np.float64), X)
    assert np.allclose(out_raw, out_n * sd_y + mu_y, rtol=1e-5, atol=1e-5)


def test_feature_oracle_invariants():
    """The feature restatement: zero rows for fixed vertices, unit RMS of the
    18 displacement-type entries, invariance of the 1-ring columns under a
    rigid translation, and the rest-state row (only gravity terms)."""
    from warpvbd_b200 import scenes
    s = scenes.cantilever(10, 2, 2)
    X, T = s.vertices, s.tets
    rng = np.random.default_rng(0)
    x = X + 1e-3 * rng.normal(size=X.shape)
    v = 0.1 * rng.normal(size=X.shape)
    f = mo.features(X, T, s.youngs, s.poisson, s.density, s.active, x, v, 1e-3, (0, 0, -9.81))
    solved = f[:, 23] > 0
    assert np.array_equal(solved, s.active)
    assert np.all(f[~solved] == 0)
    assert np.allclose(np.sqrt((f[solved, :18] ** 2).mean(1)), 1.0)
    f2 = mo.features(X, T, s.youngs, s.poisson, s.density, s.active, x + 0.3, v, 1e-3,
                     (0, 0, -9.81))
    assert np.allclose(f2, f, atol=1e-9)
    r = mo.features(X, T, s.youngs, s.poisson, s.density, s.active, X, 0 * X, 1e-3,
                    (0, 0, -9.81))[solved]
    assert np.allclose(r[:, 0:3], r[:, 15:18]) and np.all(r[:, 3:15] == 0)
    assert np.allclose(r[:, 20] * 20, np.bincount(T.reshape(-1), minlength=len(X))[solved])
