"""Mesh setup on the GPU (GPU tests): the greedy colouring computed by
Jones-Plassmann rounds with the vertex index as priority equals the
reference's sequential pass bit for bit -- against the colourings the
reference's own coloring.py produced (tests/golden) -- and a solver built
with it steps exactly like one built with the host colouring."""
import hashlib
import time

import numpy as np
import pytest

from warpvbd_b200 import scenes
from warpvbd_b200.coloring import color_tets

pytestmark = pytest.mark.gpu


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_gpu_coloring_matches_reference_goldens(golden, golden_hashes):
    names = sorted({k.split("/")[0] for k in golden.files if k.endswith("/coloring")})
    assert names
    for name in names:
        col = color_tets(golden[f"{name}/tets"], device=0)
        assert np.array_equal(col, golden[f"{name}/coloring"]), name
        assert _sha(col.astype(np.int32)) == golden_hashes[name]["coloring_sha256"], name


@pytest.mark.parametrize("n", [160, 320])
def test_gpu_coloring_of_large_cantilevers(golden_hashes, n):
    """The large cantilevers, whose reference colourings are committed as
    hashes: the GPU colouring hashes the same and equals the host pass."""
    s = scenes.cantilever(n)
    color_tets(scenes.cantilever(20).tets, device=0)  # context and module load
    t0 = time.perf_counter()
    host = color_tets(s.tets)
    t1 = time.perf_counter()
    gpu = color_tets(s.tets, device=0)
    t2 = time.perf_counter()
    print(f"cantilever {n}: host colouring {1e3 * (t1 - t0):.1f} ms, GPU {1e3 * (t2 - t1):.1f} ms")
    assert np.array_equal(host, gpu)
    key = f"cantilever_{n}"
    if key in golden_hashes:
        assert _sha(gpu.astype(np.int32)) == golden_hashes[key]["coloring_sha256"]


def test_solvers_built_with_gpu_setup_step_identically():
    from warpvbd_b200 import BatchedVBDSolver, VBDSolver
    s = scenes.cantilever(40)
    a = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000)
    b = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
                  gpu_setup=True)
    assert np.array_equal(a.color_groups, b.color_groups)
    for _ in range(5):
        xa = a.step(a.old_positions, 1e-3).numpy()
        xb = b.step(b.old_positions, 1e-3).numpy()
        assert a.last_iterations == b.last_iterations
        assert np.array_equal(xa, xb)
    envs = scenes.env_batch(12, seed=5)
    c = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
    d = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, gpu_setup=True)
    for _ in range(5):
        assert np.array_equal(c.step(1e-3), d.step(1e-3))
    assert np.array_equal(c.positions(), d.positions())
