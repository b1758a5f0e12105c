"""The autotuner's search and cache (CPU; the GPU measurement is covered in
tests/test_gpu_autotune.py)."""
import math

import numpy as np

from warpvbd_b200 import autotune


def test_coordinate_descent_finds_the_separable_optimum_once_per_config():
    space = {"a": [1, 2, 3, 4], "b": [10, 20, 30], "c": [False, True]}
    calls = []

    def cost(cfg):
        calls.append(dict(cfg))
        return (cfg["a"] - 3) ** 2 + abs(cfg["b"] - 20) / 10 + (0.5 if cfg["c"] else 0.0)

    best, c, log = autotune.coordinate_descent(space, cost)
    assert best == {"a": 3, "b": 20, "c": False} and c == 0.0
    keys = [tuple(sorted(d.items())) for d in calls]
    assert len(keys) == len(set(keys)) == len(log)


def test_unbuildable_candidates_are_skipped():
    space = {"tpv": [2, 4, 8], "cluster": [1, 16]}

    def cost(cfg):
        return math.inf if cfg["cluster"] == 16 else {2: 3.0, 4: 1.0, 8: 2.0}[cfg["tpv"]]

    best, c, _ = autotune.coordinate_descent(space, cost)
    assert best == {"tpv": 4, "cluster": 1} and c == 1.0


def test_search_families_picks_the_best_family():
    spaces = {"block": {"tpv": [2, 4]}, "persist": {"tpv": [2, 4], "block_threads": [256, 512]}}

    def cost(cfg):
        base = {"block": 5.0, "persist": 3.0}[cfg["mode"]]
        return base - (cfg["tpv"] == 4) - 0.5 * (cfg.get("block_threads") == 512)

    best, c, log = autotune.search_families(spaces, cost)
    assert best == {"mode": "persist", "tpv": 4, "block_threads": 512} and c == 1.5
    assert {d["mode"] for d, _ in log} == {"block", "persist"}


def test_cache_roundtrip_and_key_sensitivity(tmp_path):
    T = np.arange(8, dtype=np.int32).reshape(2, 4)
    X = np.zeros((8, 3))
    k1 = autotune.mesh_key("single", T, X, None, "snh", "mixed", "GPU")
    assert k1 == autotune.mesh_key("single", T.copy(), X.copy(), None, "snh", "mixed", "GPU")
    assert k1 != autotune.mesh_key("single", T, X, None, "stvk", "mixed", "GPU")
    assert k1 != autotune.mesh_key("single", T, X + 1.0, None, "snh", "mixed", "GPU")
    path = str(tmp_path / "cache.json")
    assert autotune.lookup(k1, path) is None
    cfg = {"mode": "persist", "tpv": 4, "block_threads": 256, "cluster": 0, "order_index": False}
    autotune.store(k1, cfg, {"ms_per_sweep": 0.05}, path)
    assert autotune.lookup(k1, path) == cfg


def test_committed_table_is_valid_json():
    import json
    import os
    if os.path.exists(autotune.PACKAGE_TABLE):
        d = json.load(open(autotune.PACKAGE_TABLE))
        for ent in d.values():
            assert ent["config"]["tpv"] in (0, 2, 4, 8, 16)


def test_timeline_summary_on_a_synthetic_trace():
    """The step-timeline report: blocks per SM from overlapping records, the
    busy fraction and the per-class cost, on a hand-made two-SM trace."""
    import numpy as np
    from warpvbd_b200 import timeline
    tl = {"start_ns": np.array([0, 0, 50, 0]), "end_ns": np.array([100, 50, 100, 100]),
          "env": np.array([0, 1, 2, 3]), "rank": np.array([0, 0, 0, 0]),
          "sm": np.array([0, 1, 1, 0]), "sweeps": np.array([2, 1, 1, 1]),
          "launch": np.array([1, 1, 1, 1])}
    assert timeline.blocks_per_sm(tl) == 2
    assert timeline.busy_fraction(tl, 4) == 300 / 400
    rows, cost = timeline.summarize([{"timeline": tl, "iters": np.array([2, 1, 1, 1]),
                                      "kernel_ms": 0.1}], np.array([10.0, 5, 5, 10]), 4)
    assert rows[0]["blocks"] == 4 and rows[0]["last"][0] in (0, 2, 3)
    assert abs(cost["single"] - 300 / (20 + 5 + 5 + 10)) < 1e-12
