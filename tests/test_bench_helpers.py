"""The bench's bookkeeping (CPU): algorithmic bytes per sweep and per
warm-start check, the sweep histogram and the tip-error summary."""
import importlib.util
import os

import numpy as np

from warpvbd_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(HERE, "..", "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_sweep_bytes_match_the_per_vertex_model():
    b = _bench()
    s = scenes.cantilever(20)
    total, solved, slots = b.sweep_bytes(s)
    k = np.bincount(s.tets.reshape(-1), minlength=s.n_vertices)
    act = s.active & (k > 0)
    assert solved == int(act.sum()) == 180
    assert slots == int(k[act].sum())
    assert total == 44 * solved + 104 * slots
    # 160x16x16: the per-sweep figure the roofline uses (87.0 MB)
    big = b.sweep_bytes(scenes.cantilever(160))[0]
    assert abs(big - 86.97e6) < 0.01e6


def test_warm_stage_bytes_count_each_tet_once():
    b = _bench()
    s = scenes.cantilever(20)
    k = np.bincount(s.tets.reshape(-1), minlength=s.n_vertices)
    act = s.active & (k > 0)
    n_tets = int(act[s.tets].any(axis=1).sum())
    assert b.warm_stage_bytes(s) == 176 * n_tets + 44 * int(act.sum())
    # far less than a sweep (every tet is read four times there)
    assert b.warm_stage_bytes(s) < 0.5 * b.sweep_bytes(s)[0]


def test_sweep_histogram_bins():
    b = _bench()
    h = b.sweep_histogram(np.array([[1, 3, 4], [7, 8, 1000]]))
    assert h["edges"][0] == 1 and h["edges"][-1] == b.MAX_ITER + 1
    assert h["counts"][:4] == [1, 1, 2, 1] and sum(h["counts"]) == 6


def test_tip_error_normalises_by_the_largest_plain_displacement():
    b = _bench()
    plain = np.zeros((3, 2, 3))
    plain[:, 0, 2] = [-1.0, -2.0, -4.0]     # env 0 swings to 4
    plain[:, 1, 2] = [-0.5, -0.5, -0.5]
    warm = plain.copy()
    warm[2, 0, 2] += 0.04                   # 1e-2 of env 0's largest displacement
    r = b.tip_error(warm, plain, "fp64")
    assert abs(r["max"] - 0.01) < 1e-12
    assert r["median"] == 0.0
    assert r["max_by_checkpoint"] == [0.0, 0.0, r["max"]]
    assert r["within_target"] is False and r["target"] == 1e-4
