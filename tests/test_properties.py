"""Property tests (hypothesis) of the host-side pieces on random voxel shapes:
the mesher, the native greedy colouring against the reference-shaped Python
pass, the OBJ surface export and the multi-GPU partition.  CPU only."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from warpvbd_b200 import coloring, distributed, io, mesh

SETTINGS = dict(max_examples=25, deadline=None,
                suppress_health_check=[HealthCheck.too_slow])


@st.composite
def voxel_shapes(draw):
    """A random voxel occupancy of up to 5 x 4 x 4 with at least one voxel."""
    nx = draw(st.integers(1, 5))
    ny = draw(st.integers(1, 4))
    nz = draw(st.integers(1, 4))
    bits = draw(st.lists(st.booleans(), min_size=nx * ny * nz, max_size=nx * ny * nz))
    vox = np.array(bits, bool).reshape(nx, ny, nz)
    if not vox.any():
        vox[draw(st.integers(0, nx - 1)), 0, 0] = True
    return vox


def _tet_mesh(vox, h=0.1):
    X, hexes = mesh.voxel2hex(vox, h, h, h)
    return np.asarray(X, np.float64), np.asarray(mesh.hex2tets(hexes), np.int64).reshape(-1, 4)


@settings(**SETTINGS)
@given(voxel_shapes())
def test_mesher_tets_are_positive_and_fill_the_voxels(vox):
    X, T = _tet_mesh(vox)
    a, b, c, d = (X[T[:, i]] for i in range(4))
    vol = np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a) / 6.0
    assert np.all(np.abs(vol) > 1e-12)
    assert abs(np.abs(vol).sum() - vox.sum() * 0.1 ** 3) < 1e-12
    assert T.min() >= 0 and T.max() < len(X)
    # every vertex belongs to some tet
    assert np.array_equal(np.unique(T), np.arange(len(X)))


@settings(**SETTINGS)
@given(voxel_shapes())
def test_native_colouring_is_the_reference_greedy_pass(vox):
    _, T = _tet_mesh(vox)
    col = coloring.color_tets(T)
    # same colours as the reference-shaped Python pass (coloring.py:24-72)
    adj, _ = coloring.compute_adjacency_dict(T)
    ref, _ = coloring.graph_coloring(adj)
    assert np.array_equal(np.asarray(col), np.asarray(ref))
    # vertices of one colour share no tet: their updates cannot race
    for t in T:
        assert len(set(col[t].tolist())) == 4


@settings(**SETTINGS)
@given(voxel_shapes())
def test_surface_covers_the_exposed_voxel_faces_outward(vox):
    """The reference mesher splits every hex the same way, so neighbouring
    hexes' shared faces get crossing diagonals and those faces stay in the
    surface too (tet2obj keeps a face seen once); the exposed faces of the
    voxel union must be covered exactly, each triangle facing out."""
    h = 0.1
    X, T = _tet_mesh(vox, h)
    V, F = io.tet_surface(X, T)
    filled = np.pad(vox, 1)
    covered = 0.0
    for f in F:
        p = V[f]
        n = np.cross(p[1] - p[0], p[2] - p[0])
        axis = int(np.argmax(np.abs(n)))
        if not np.allclose(p[:, axis], p[0, axis]):
            continue  # a diagonal face inside a hex
        # the plane at index k separates voxels k - 1 and k along `axis`
        # (padded indices k and k + 1)
        c = p.mean(0) / h
        k = int(round(p[0, axis] / h))
        idx = [int(np.floor(c[i])) + 1 for i in range(3)]
        idx[axis] = k + 1
        hi_side = bool(filled[tuple(idx)])
        idx[axis] = k
        lo_side = bool(filled[tuple(idx)])
        if hi_side == lo_side:
            continue  # an interior face
        covered += 0.5 * np.linalg.norm(n)
        # outward: the normal points from the filled side to the empty one
        assert (n[axis] > 0) == lo_side
    exposed = sum(np.abs(np.diff(filled.astype(int), axis=a)).sum() for a in range(3))
    assert abs(covered - exposed * h * h) < 1e-9


@settings(**SETTINGS)
@given(st.lists(st.floats(0.1, 100.0), min_size=1, max_size=60), st.integers(1, 9))
def test_partition_is_a_balanced_cover(weights, n_parts):
    parts = distributed.partition(weights, n_parts)
    assert len(parts) == n_parts
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(weights)))
    loads = [sum(weights[i] for i in p) for p in parts]
    # longest-first greedy: no part exceeds the mean load by more than one item
    assert max(loads) <= sum(weights) / n_parts + max(weights) + 1e-9
