"""Output formats (CPU): the OBJ surface export against the reference's own
tet2obj (golden fixtures from tests/golden/make_obj_golden.py), and the tip
trajectory CSV / npz files."""
import os

import numpy as np
import pytest

from warpvbd_b200 import io, scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["cantilever_20", "massspring_7_5", "ragged_6x5x4"])
def test_surface_matches_reference_tet2obj(name):
    meshes = np.load(os.path.join(GOLDEN, "meshes.npz"))
    surf = np.load(os.path.join(GOLDEN, "surfaces.npz"))
    v, f = io.tet_surface(meshes[f"{name}/vertices"], meshes[f"{name}/tets"])
    assert np.array_equal(v, surf[f"{name}/vertices"])
    assert np.array_equal(f, surf[f"{name}/faces"])


def test_write_obj_format(tmp_path):
    s = scenes.cantilever(20)
    path = str(tmp_path / "beam.obj")
    v, f = io.write_obj(path, s.vertices, s.tets)
    lines = open(path).read().splitlines()
    vs = [ln for ln in lines if ln.startswith("v ")]
    fs = [ln for ln in lines if ln.startswith("f ")]
    assert len(vs) == len(v) and len(fs) == len(f)
    idx = np.array([[int(t) for t in ln.split()[1:]] for ln in fs])
    assert idx.min() == 1 and idx.max() == len(v)
    assert np.allclose(np.array([[float(t) for t in ln.split()[1:]] for ln in vs]), v)


def test_single_tet_surface_is_outward():
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    v, f = io.tet_surface(X, np.array([[0, 1, 2, 3]]))
    assert f.shape == (4, 3)
    c = v.mean(0)
    for t in f:
        a, b, d = v[t]
        n = np.cross(b - a, d - a)
        assert n.dot((a + b + d) / 3 - c) > 0


def test_tip_csv_and_npz_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    tips = rng.normal(size=(7, 3))
    p = str(tmp_path / "tip.csv")
    io.save_tip_csv(p, tips)
    assert np.allclose(np.loadtxt(p, delimiter=","), tips)
    per_env = [rng.normal(size=(5, 3)), rng.normal(size=(5, 3))]
    q = str(tmp_path / "tips.npz")
    io.save_tip_npz(q, per_env)
    d = np.load(q)
    assert sorted(d.keys()) == ["0", "1"] and np.allclose(d["1"], per_env[1])
    s = scenes.cantilever(20)
    assert np.allclose(io.tip_positions(s.vertices, s.tip), s.vertices[s.tip].mean(0))


def test_state_checkpoint_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    x, v = rng.normal(size=(17, 3)), rng.normal(size=(17, 3))
    p = tmp_path / "state.npz"
    io.save_state(p, x, v, step=np.int64(12))
    x2, v2, extra = io.load_state(p)
    assert np.array_equal(x, x2) and np.array_equal(v, v2) and int(extra["step"]) == 12


def test_step_log_jsonl(tmp_path):
    from warpvbd_b200 import metrics
    p = str(tmp_path / "run.jsonl")
    log = metrics.StepLog(p, n_solved=[100, 50], dt=1e-3)
    log.record([10, 20], 0.002)
    log.record([5, 6], 0.001, note="x")
    log.close()
    rows = metrics.read(p)
    assert [r["step"] for r in rows] == [1, 2]
    assert rows[0]["sweeps_max"] == 20 and rows[0]["sweeps_mean"] == 15
    assert abs(rows[0]["sim_s_per_wall_s"] - 1.0) < 1e-12       # 2 envs x 1 ms / 2 ms
    assert abs(rows[0]["vertex_updates_per_s"] - (100 * 10 + 50 * 20) / 0.002) < 1e-6
    assert abs(rows[1]["run_sim_s_per_wall_s"] - 2 * 2e-3 / 0.003) < 1e-12
    assert rows[1]["note"] == "x"
