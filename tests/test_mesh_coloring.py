"""Mesher and colouring against the reference's own outputs (tests/golden).

The fixtures were produced by importing the reference's src/_utils.py
(voxel2hex, hex2tets) and src/coloring.py (compute_adjacency_dict,
graph_coloring) -- see tests/golden/make_golden.py.  Colour groups must be
bit-exact.
"""
import hashlib

import numpy as np
import pytest

from warpvbd_b200 import mesh, scenes
from oracle import oracle


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _scene_arrays(name, spec):
    vox_shape = tuple(spec["voxels_shape"])
    if name.startswith("cantilever"):
        n = vox_shape[0]
        s = scenes.cantilever(n)
        return s.vertices, s.tets
    if name.startswith("massspring"):
        _, cube, col = name.split("_")
        s = scenes.mass_spring(int(cube), int(col))
        return s.vertices, s.tets
    return None


SMALL = ["cantilever_20", "cantilever_40", "cantilever_80", "massspring_11_20", "massspring_7_5",
         "massspring_15_30", "massspring_9_13"]


@pytest.mark.parametrize("name", SMALL)
def test_mesher_matches_reference(name, golden):
    from tests.conftest import ROOT  # noqa: F401
    spec_vertices = golden[f"{name}/vertices"]
    spec_tets = golden[f"{name}/tets"]
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "hashes.json")) as f:
        spec = json.load(f)[name]
    X, T = _scene_arrays(name, spec)
    assert np.array_equal(X, spec_vertices)          # bit-exact float64
    assert np.array_equal(T, spec_tets)


def test_ragged_voxels_match_reference(golden):
    vox = golden["ragged_6x5x4/voxels"]
    X, H = mesh.voxel2hex(vox, 0.02, 0.03, 0.05)
    T = mesh.hex2tets(H).astype(np.int32)
    assert np.array_equal(X, golden["ragged_6x5x4/vertices"])
    assert np.array_equal(T, golden["ragged_6x5x4/tets"])


@pytest.mark.parametrize("name", ["cantilever_160", "cantilever_320"])
def test_large_meshes_hash_match(name, golden_hashes):
    spec = golden_hashes[name]
    X, T = _scene_arrays(name, spec)
    assert X.shape[0] == spec["n_vertices"] and T.shape[0] == spec["n_tets"]
    assert sha(X) == spec["vertices_sha256"]
    assert sha(T.astype(np.int32)) == spec["tets_sha256"]


ALL_SMALL = SMALL + ["ragged_6x5x4"]


@pytest.mark.parametrize("name", ALL_SMALL)
def test_oracle_coloring_bit_exact(name, golden):
    col = oracle.graph_coloring(golden[f"{name}/tets"])
    assert np.array_equal(col, golden[f"{name}/coloring"])


@pytest.mark.parametrize("name", ALL_SMALL)
def test_native_coloring_bit_exact(name, golden):
    from warpvbd_b200.coloring import color_tets
    col = color_tets(golden[f"{name}/tets"])
    assert np.array_equal(col, golden[f"{name}/coloring"])


@pytest.mark.parametrize("name", ["cantilever_20", "ragged_6x5x4", "massspring_7_5"])
def test_reference_shaped_coloring_api(name, golden):
    from warpvbd_b200.coloring import compute_adjacency_dict, graph_coloring, color_groups_dict
    adj, deg = compute_adjacency_dict(golden[f"{name}/tets"])
    col, groups = graph_coloring(adj)
    assert np.array_equal(col, golden[f"{name}/coloring"])
    assert groups == color_groups_dict(golden[f"{name}/coloring"])


@pytest.mark.parametrize("name", ["cantilever_160", "cantilever_320"])
def test_native_coloring_large_hash(name, golden_hashes):
    from warpvbd_b200.coloring import color_tets
    spec = golden_hashes[name]
    _, T = _scene_arrays(name, spec)
    col = color_tets(T)
    assert sha(col.astype(np.int32)) == spec["coloring_sha256"]
    assert np.bincount(col).tolist() == spec["color_group_sizes"]


def test_coloring_is_valid_and_groups_ascending(golden):
    T = golden["massspring_11_20/tets"]
    col = oracle.graph_coloring(T)
    for t in T:
        assert len(set(col[t].tolist())) == 4     # no two vertices of a tet share a colour


def test_env_batch_seeded_and_uneven():
    a = scenes.env_batch(8, seed=3)
    b = scenes.env_batch(8, seed=3)
    assert [e.n_vertices for e in a] == [e.n_vertices for e in b]
    assert len({e.n_vertices for e in a}) > 1
    for e in a:
        assert 7 <= e.meta["cube"] <= 15 and 5 <= e.meta["column"] <= 30
        assert 1e5 <= e.youngs[0] <= 1e6 and 0.35 <= e.poisson[0] <= 0.48
        assert e.active.sum() == e.n_vertices - 4      # the column's top face is fixed
