"""The autotuner on the GPU: it measures real candidates, caches the winner,
and the tuned solver still matches the FP64 oracle."""
import time

import numpy as np
import pytest

from oracle import oracle
from warpvbd_b200 import autotune, scenes

pytestmark = pytest.mark.gpu

SMALL = {"block": {"tpv": [4, 8], "cluster": [1, 2]},
         "persist": {"tpv": [4, 8], "block_threads": [256]}}


def test_tune_single_measures_caches_and_the_result_matches_the_oracle(tmp_path):
    from warpvbd_b200 import VBDSolver
    s = scenes.cantilever(20)
    path = str(tmp_path / "tune.json")
    cfg = autotune.tune_single(s.solver_kwargs(), spaces=SMALL, cache_path=path, refresh=True)
    assert cfg["mode"] in ("block", "persist") and cfg["tpv"] in (4, 8)
    t0 = time.perf_counter()
    assert autotune.tune_single(s.solver_kwargs(), spaces=SMALL, cache_path=path) == cfg
    assert time.perf_counter() - t0 < 1.0        # served from the cache, nothing measured
    gpu = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7, max_iter=1000,
                    **cfg)
    orc = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                              max_iter=1000, guarded=True)
    D = float(np.linalg.norm(s.vertices.max(0) - s.vertices.min(0)))
    for _ in range(50):
        xg = gpu.step(gpu.old_positions, 1e-3).numpy()
        xo = orc.step(None, 1e-3)
    assert np.abs(xg - xo).max() / D < 1e-5


def test_tune_batched_and_tune_flag(tmp_path, monkeypatch):
    from warpvbd_b200 import BatchedVBDSolver
    monkeypatch.setenv("WARPVBD_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    envs = scenes.env_batch(6, seed=3)
    spaces = {"block": {"tpv": [4, 2], "cluster": [1, 2]}}
    cfg = autotune.tune_batched(envs, spaces=spaces, refresh=True)
    assert cfg["tpv"] in (2, 4) and cfg["cluster"] in (1, 2) and "mode" not in cfg
    tuned = BatchedVBDSolver(envs, tune=True)     # cache hit: the same shape
    assert tuned.info()["tpv"] == cfg["tpv"]
    plain = BatchedVBDSolver(envs, tpv=4, cluster=1)
    for _ in range(10):
        it_a = tuned.step(1e-3)
        it_b = plain.step(1e-3)
    D = max(float(np.linalg.norm(e.vertices.max(0) - e.vertices.min(0))) for e in envs)
    assert np.abs(tuned.positions() - plain.positions()).max() / D < 1e-6
