"""The FP64 oracle against trajectories of the reference's own solver code
(CPU tests).

``tests/golden/ref_trajectories.npz`` was produced by running the
reference's unchanged ``src/vbd_solver.py`` (mmichelis/WarpVBD) through a
pure-Python stand-in for Warp (``tests/golden/make_ref_trajectories.py``).
The oracle restates the same algorithm in C; both compute in IEEE double
precision, so they agree to rounding: the same sweep count at every step and
positions within 1e-12 of the bounding-box diagonal (measured: about 1e-16).
Together with the GPU tests this pins the CUDA solver to the reference
through the oracle and directly.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["cantilever20_snh", "cantilever20_stvk", "cantilever20_damped",
         "cantilever20_maxiter3", "massspring5_6"]


@pytest.fixture(scope="module")
def ref():
    # meshes of a few hundred vertices: one thread is fastest
    oracle.set_threads(1)
    return np.load(os.path.join(HERE, "golden", "ref_trajectories.npz"))


def _diag(X):
    return float(np.linalg.norm(X.max(0) - X.min(0)))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_trajectory(ref, name):
    p = json.loads(str(ref[f"{name}/params"]))
    X, T, act = ref[f"{name}/vertices"], ref[f"{name}/tets"], ref[f"{name}/active"]
    n = T.shape[0]
    o = oracle.OracleSolver(X, T, np.full(n, p["rho"]), np.full(n, p["E"]), np.full(n, p["nu"]),
                            damping_coefficient=p["kd"], active_mask=act, dx_tol=p["tol"],
                            max_iter=p["max_iter"], material=p["material"])
    # the tables the reference built (colouring.py order, ascending adjacency)
    assert np.array_equal(o.color_groups, ref[f"{name}/color_groups"])
    assert np.array_equal(o.adj_v2e, ref[f"{name}/adj_v2e"])
    rec = ref[f"{name}/rec_steps"].tolist()
    pos = ref[f"{name}/positions"]
    sweeps, warned = ref[f"{name}/sweeps"], ref[f"{name}/warned"]
    D = _diag(X)
    worst, j = 0.0, 0
    for k in range(1, len(sweeps) + 1):
        x = o.step(None, p["dt"])
        assert o.last_iterations == sweeps[k - 1], (k, o.last_iterations, sweeps[k - 1])
        assert o.warned == bool(warned[k - 1])
        if k in rec:
            worst = max(worst, np.abs(x - pos[j]).max() / D)
            j += 1
    assert j == len(rec)
    assert worst < 1e-12, worst


def test_reference_fixture_covers_the_configured_cantilever(ref):
    """The golden SNH case is the configured 20x2x2 cantilever, 300 steps of
    1 ms at tol 1e-7, and its mesh is the product mesher's (pinned bit-exact
    to the reference's mesher by meshes.npz)."""
    from warpvbd_b200 import scenes
    p = json.loads(str(ref["cantilever20_snh/params"]))
    assert (p["steps"], p["dt"], p["tol"], p["max_iter"], p["E"], p["nu"], p["rho"]) == \
        (300, 1e-3, 1e-7, 1000, 1e6, 0.45, 1000.0)
    s = scenes.cantilever(20)
    assert np.array_equal(s.vertices, ref["cantilever20_snh/vertices"])
    assert np.array_equal(s.tets, ref["cantilever20_snh/tets"])
    assert np.array_equal(s.active, ref["cantilever20_snh/active"])
    assert ref["cantilever20_maxiter3/warned"].all()
    assert not ref["cantilever20_snh/warned"].any()


def test_long_fixture_starts_like_the_oracle():
    """The first steps of the long mass-spring fixture recomputed here."""
    from warpvbd_b200 import scenes
    oracle.set_threads(1)
    long = np.load(os.path.join(HERE, "golden", "oracle_long.npz"))
    s = scenes.mass_spring(11, 20)
    o = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                            max_iter=1000, guarded=True)
    for k in range(15):
        x = o.step(None, 1e-3)
        assert o.last_iterations == long["c3/sweeps"][k]
        d = (x[s.tip] - s.vertices[s.tip]).mean(0)
        assert np.allclose(d, long["c3/tip"][k], rtol=1e-12, atol=1e-15)
