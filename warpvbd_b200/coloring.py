"""Greedy vertex colouring of a tet mesh (reference: mmichelis/WarpVBD src/coloring.py).

``color_tets`` runs the native colouring of libvbd_b200.so (vbd_graph_coloring),
the same greedy pass as the reference's ``graph_coloring`` (coloring.py:40-72)
over the adjacency of ``compute_adjacency_dict`` (coloring.py:24-38): vertices
in index order, each taking the smallest colour not used by an
already-coloured vertex that shares a tet.  The reference-shaped
``compute_adjacency_dict`` / ``graph_coloring`` pair is kept for callers of
that interface.
"""
import ctypes

import numpy as np

from . import _lib

MAX_COLORS = 256  # coloring.py:50


def color_tets(elements, device=None):
    """Per-vertex colour (int32[max(elements)+1]) of the greedy colouring.
    `device` (a CUDA device ordinal): compute it on that GPU with
    vbd_graph_coloring_gpu -- Jones-Plassmann rounds with the vertex index as
    priority, which give exactly the sequential pass's colours."""
    tets = _lib.i32(np.asarray(elements)).reshape(-1, 4)
    nv = int(tets.max()) + 1 if tets.size else 0
    out = np.empty(max(nv, 1), dtype=np.int32)
    n_v, n_c = ctypes.c_int(0), ctypes.c_int(0)
    L = _lib.load()
    if device is None:
        st = L.vbd_graph_coloring(_lib.ptr(tets, "i"), tets.shape[0], _lib.ptr(out, "i"),
                                  ctypes.byref(n_v), ctypes.byref(n_c))
    else:
        st = L.vbd_graph_coloring_gpu(_lib.ptr(tets, "i"), tets.shape[0], _lib.ptr(out, "i"),
                                      ctypes.byref(n_v), ctypes.byref(n_c), int(device))
    if st == _lib.ERR_TOO_MANY_COLORS:
        raise AssertionError("Exceeded maximum number of colors")
    _lib.check(st, "vbd_graph_coloring")
    return out[:n_v.value]


def color_groups_dict(coloring):
    """{colour: [vertex ids ascending]} as returned by the reference's graph_coloring."""
    coloring = np.asarray(coloring)
    return {int(c): np.nonzero(coloring == c)[0].tolist()
            for c in range(int(coloring.max()) + 1 if coloring.size else 0)}


def color_groups_table(coloring):
    """int32 [n_colors, max_group], -1 padded (vbd_solver.py:476-483)."""
    groups = color_groups_dict(coloring)
    mg = max((len(g) for g in groups.values()), default=0)
    out = np.full((len(groups), mg), -1, dtype=np.int32)
    for c, g in groups.items():
        out[c, :len(g)] = g
    return out


def compute_adjacency_dict(elements):
    """(adjacency {v: set of 1-ring neighbours}, maximal degree) -- coloring.py:24-38."""
    tets = np.asarray(elements)
    num_vertices = int(tets.max()) + 1
    adjacency = {i: set() for i in range(num_vertices)}
    maximal_degree = 0
    for ele in tets.tolist():
        for i, a in enumerate(ele):
            for b in ele[i + 1:]:
                adjacency[a].add(b)
                adjacency[b].add(a)
            maximal_degree = max(maximal_degree, len(adjacency[a]))
    return adjacency, maximal_degree


def graph_coloring(adjacency):
    """(coloring, color_groups) for an adjacency dict -- coloring.py:40-72."""
    n = len(adjacency)
    coloring = -np.ones(n, dtype=int)
    groups = {}
    for v in range(n):
        used = {coloring[u] for u in adjacency[v] if coloring[u] != -1}
        for c in range(MAX_COLORS):
            if c not in used:
                coloring[v] = c
                groups.setdefault(c, []).append(v)
                break
        else:
            raise AssertionError("Exceeded maximum number of colors")
    return coloring, groups
