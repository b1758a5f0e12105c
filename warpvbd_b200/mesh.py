"""Voxel -> hexahedron -> tetrahedron mesher.

Same numbering and split as the reference's mesher (mmichelis/WarpVBD
src/_utils.py:35-108), vectorised with numpy instead of Python loops:

* ``voxel2hex`` (reference ``_utils.py:35-89``): a vertex exists at every
  lattice corner touched by a filled voxel; vertices are numbered with ``i``
  fastest, then ``j``, then ``k``; coordinates are ``(dx*i, dy*j, dz*k)``;
  hexes are listed in the same k/j/i order with the VTK corner order
  0:(i,j,k) 1:(i+1,j,k) 2:(i+1,j+1,k) 3:(i,j+1,k) and 4-7 the same at k+1.
* ``hex2tets`` (reference ``_utils.py:92-108``): every hex is split into the
  same five tets (0,1,3,4) (1,2,3,6) (1,4,5,6) (3,4,6,7) (1,3,4,6).

Both are pinned bit-exact against the reference by tests/golden.
"""
import numpy as np

# local hex corner offsets (di, dj, dk) in VTK order
_HEX_CORNERS = np.array([
    (0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
    (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1),
], dtype=np.int64)

# five-tet split of one hex, as hex-corner indices
HEX_TO_TETS = np.array([
    (0, 1, 3, 4),
    (1, 2, 3, 6),
    (1, 4, 5, 6),
    (3, 4, 6, 7),
    (1, 3, 4, 6),
], dtype=np.int64)


def voxel2hex(voxels, dx, dy, dz):
    """Filled voxels -> (vertices float64[V,3], hexes int64[H,8])."""
    vox = np.asarray(voxels).astype(bool)
    nx, ny, nz = vox.shape
    flag = np.zeros((nx + 1, ny + 1, nz + 1), dtype=bool)
    for di, dj, dk in _HEX_CORNERS:
        flag[di:di + nx, dj:dj + ny, dk:dk + nz] |= vox
    # number vertices with i fastest, then j, then k: iterate in (k, j, i) order
    order = np.transpose(flag, (2, 1, 0))  # [k, j, i]
    kk, jj, ii = np.nonzero(order)
    index = np.full((nx + 1, ny + 1, nz + 1), -1, dtype=np.int64)
    index[ii, jj, kk] = np.arange(ii.size, dtype=np.int64)
    vertices = np.stack([dx * ii.astype(np.float64), dy * jj.astype(np.float64),
                         dz * kk.astype(np.float64)], axis=1)
    # reference multiplies a Python float by a Python int; for exact-integer
    # conversions float64(i)*dx is the same IEEE product
    hk, hj, hi = np.nonzero(np.transpose(vox, (2, 1, 0)))
    hexes = np.stack([index[hi + di, hj + dj, hk + dk] for di, dj, dk in _HEX_CORNERS], axis=1)
    return vertices, hexes


def hex2tets(hex_elements):
    """hexes int[H,8] -> tets int64[5H,4], five tets per hex in the fixed split."""
    h = np.asarray(hex_elements)
    return h[:, HEX_TO_TETS].reshape(-1, 4).astype(np.int64)
