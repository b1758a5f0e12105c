"""Edge cases of the CUDA solver against the FP64 oracle (GPU, through the C
ABI): an environment with every vertex fixed, a one-tet environment and a
vertex in no tet inside a batch, a batch of one against the single-mesh
solver, and a vertex of valence 40 (beyond the reference's 32-entry
adjacency rows: here a vertex's slots stream past the prefetched steps)."""
import numpy as np
import pytest

from oracle import oracle
from warpvbd_b200 import scenes
from warpvbd_b200.scenes import Scene

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5


def _diag(X):
    return float(np.linalg.norm(X.max(0) - X.min(0))) or 1.0


def _scene(X, T, active, youngs=1e5, name="edge"):
    T = np.asarray(T, np.int32).reshape(-1, 4)
    n_t = T.shape[0]
    return Scene(name=name, vertices=np.asarray(X, np.float64), tets=T,
                 active=np.asarray(active, bool), tip=np.arange(min(4, len(X))),
                 density=np.full(n_t, 1000.0), youngs=np.full(n_t, youngs),
                 poisson=np.full(n_t, 0.4))


def _one_tet():
    X = np.array([[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0], [0, 0, 0.1]], float)
    return _scene(X, [[0, 1, 2, 3]], [False, True, True, True], name="one tet")


def _fan(n=40, h=0.05):
    """A centre vertex on n tets: ring vertices around it, one apex above;
    the ring and apex fixed except every other ring vertex."""
    ang = 2 * np.pi * np.arange(n) / n
    ring = np.stack([h * np.cos(ang), h * np.sin(ang), np.zeros(n)], 1)
    X = np.concatenate([[[0, 0, 0]], ring, [[0, 0, h]]])
    T = [[0, 1 + i, 1 + (i + 1) % n, n + 1] for i in range(n)]
    active = np.zeros(n + 2, bool)
    active[0] = True
    active[1::2] = True
    active[n + 1] = False
    return _scene(X, T, active, name="fan")


def _oracle_run(s, steps, dt=1e-3):
    o = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                            max_iter=1000, guarded=True)
    xs, its = [], []
    for _ in range(steps):
        xs.append(o.step(None, dt).copy())
        its.append(o.last_iterations)
    return xs, its


def test_batch_with_fixed_one_tet_and_free_vertex_environments():
    from warpvbd_b200 import BatchedVBDSolver
    base = scenes.mass_spring(7, 5)
    fixed = scenes.mass_spring(7, 5)
    fixed = _scene(fixed.vertices, fixed.tets, np.zeros(fixed.n_vertices, bool), name="fixed")
    # a vertex in no tet, active: it follows the inertia guess (free fall)
    one = _one_tet()
    loose = _scene(np.concatenate([one.vertices, [[0.3, 0.3, 0.3]]]), one.tets,
                   np.concatenate([one.active, [True]]), name="loose vertex")
    envs = [base, fixed, one, loose]
    b = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    refs = [_oracle_run(e, 10) for e in envs]
    for k in range(10):
        b.step(1e-3)
        x = b.positions()
        for e, env in enumerate(envs):
            xe = x[b.env_slice(e)]
            assert np.abs(xe - refs[e][0][k]).max() / _diag(env.vertices) < POS_TOL, (k, env.name)
    x = b.positions()
    assert np.array_equal(x[b.env_slice(1)], fixed.vertices)     # nothing moves
    t = 10e-3
    free = x[b.env_slice(3)][-1]
    assert np.allclose(free, [0.3, 0.3, 0.3 - 0.5 * 9.81 * t * (t + 1e-3)], atol=1e-9)


def test_batch_of_one_equals_single_mesh_solver():
    from warpvbd_b200 import BatchedVBDSolver, VBDSolver
    s = scenes.mass_spring(9, 10)
    b = BatchedVBDSolver([s], dx_tol=1e-7, max_iter=1000, cluster=1)
    v = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
                  mode="block", cluster=1)
    for _ in range(10):
        it_b = b.step(1e-3)
        xv = v.step(v.old_positions, 1e-3).numpy()
        assert int(it_b[0]) == v.last_iterations
    assert np.abs(b.positions() - xv).max() < 1e-12


@pytest.mark.parametrize("mode", ["block", "persist", "graph"])
def test_high_valence_vertex(mode):
    """The reference refuses a vertex on more than 32 tets (its padded
    adjacency rows); so does the wrapper by default.  With
    allow_high_valence=True the 40-tet vertex is solved like any other."""
    from warpvbd_b200 import VBDSolver
    s = _fan(40)
    assert np.bincount(s.tets.reshape(-1))[0] == 40
    kw = dict(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
              mode=mode)
    strict = VBDSolver(**kw)
    with pytest.raises(AssertionError):
        strict.step(strict.old_positions, 1e-3)
    gpu = VBDSolver(**kw, allow_high_valence=True)
    xs, its = _oracle_run(s, 20)
    for k in range(20):
        x = gpu.step(gpu.old_positions, 1e-3).numpy()
        assert np.abs(x - xs[k]).max() / _diag(s.vertices) < POS_TOL, k
        assert abs(gpu.last_iterations - its[k]) <= 2
