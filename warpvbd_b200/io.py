"""Output formats of the reference's drivers, for headless inspection, and
state checkpoints.

* Tip trajectories: ``save_tip_csv`` writes the per-step tip-face mean
  positions as CSV, one ``x,y,z`` row per step (examples/run_cantilever.py:177
  stores ``np.array(tip_positions)`` with ``np.savetxt(..., delimiter=",")``);
  ``save_tip_npz`` writes one array per environment under its index as key,
  compressed (examples/run_mass_spring_parallel.py:221).
* Surface meshes: ``tet_surface`` returns the boundary triangles of a tet
  mesh and ``write_obj`` stores them as a Wavefront OBJ, following
  src/_renderer.py:539-582 (``tet2obj``): a face shared by two tets is
  interior, every other face is kept with the outward orientation of its tet
  (``fix_tet_faces``, :466-485), faces in the order the tets list them, and
  the vertices no face uses are dropped with the rest renumbered in their
  original order (``filter_unused_vertices``, :435-460).  Written here with
  array operations instead of a per-face dictionary; the golden test checks
  the output against the reference's own function.
"""
import numpy as np

# local face vertex triples of a tet, by the sign of
# cross(v1 - v0, v2 - v1) . (v3 - v0)  (negative: first row, else second)
_FACES_NEG = np.array([(0, 1, 2), (2, 1, 3), (1, 0, 3), (0, 2, 3)])
_FACES_POS = np.array([(1, 0, 2), (1, 2, 3), (0, 1, 3), (2, 0, 3)])


def tet_surface(vertices, tets):
    """(surface vertices [n, 3] float64, triangles [m, 3] int64 into them)."""
    X = np.asarray(vertices, np.float64).reshape(-1, 3)
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    if T.shape[0] == 0:
        return np.zeros((0, 3)), np.zeros((0, 3), np.int64)
    v0, v1, v2, v3 = (X[T[:, i]] for i in range(4))
    neg = np.einsum("ij,ij->i", np.cross(v1 - v0, v2 - v1), v3 - v0) < 0
    local = np.where(neg[:, None, None], _FACES_NEG[None], _FACES_POS[None])  # [T, 4, 3]
    faces = np.take_along_axis(T[:, None, :].repeat(4, axis=1), local, axis=2).reshape(-1, 3)
    # a face seen twice is interior; keep the others in the order they appear
    key = np.sort(faces, axis=1)
    _, inverse, counts = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    faces = faces[counts[inverse.reshape(-1)] == 1]
    used = np.zeros(X.shape[0], bool)
    used[faces.reshape(-1)] = True
    remap = np.full(X.shape[0], -1, np.int64)
    remap[used] = np.arange(int(used.sum()))
    return X[used], remap[faces]


def write_obj(path, vertices, tets):
    """Store the boundary surface of a tet mesh as an OBJ file (1-based
    indices); returns (surface vertices, triangles)."""
    v, f = tet_surface(vertices, tets)
    with open(path, "w") as out:
        for p in v:
            out.write("v {} {} {}\n".format(p[0], p[1], p[2]))
        for t in f:
            out.write("f {} {} {}\n".format(t[0] + 1, t[1] + 1, t[2] + 1))
    return v, f


def tip_positions(positions, tip):
    """Mean position of the tip vertices (the reference drivers' measure)."""
    return np.asarray(positions, np.float64)[np.asarray(tip)].mean(axis=0)


def save_tip_csv(path, tip_positions_per_step):
    np.savetxt(path, np.asarray(tip_positions_per_step, np.float64).reshape(-1, 3),
               delimiter=",")


def save_tip_npz(path, tip_positions_per_env):
    """`tip_positions_per_env`: sequence (or dict) of per-step tip positions
    per environment; keys are the environment indices as strings."""
    items = (tip_positions_per_env.items() if isinstance(tip_positions_per_env, dict)
             else enumerate(tip_positions_per_env))
    np.savez_compressed(path, **{str(k): np.asarray(v, np.float64) for k, v in items})


__all__ = ["tet_surface", "write_obj", "tip_positions", "save_tip_csv", "save_tip_npz",
           "save_state", "load_state"]


def save_state(path, positions, velocities, **extra):
    """Checkpoint of a solver's state (x, v) as a compressed npz (float64
    [n, 3] each; `extra` arrays are stored too, e.g. the step count).  Restore
    with load_state and the solver's set_state(positions=..., velocities=...).

    (x, v) is all a plain VBD step depends on, and a restored plain run
    continues like the uninterrupted one (same sweep counts; positions equal
    up to the rounding of x - X).  A solver with the learned warm start also
    feeds the previous step's inertia target to its network, which a fresh
    solver does not have: after a restore its first step predicts from
    (x, v) alone and may take another candidate, so a resumed warm-started run
    agrees with the uninterrupted one to the solver's tolerance (both stop
    when the update falls below dx_tol), not bit for bit."""
    np.savez_compressed(path, positions=np.asarray(positions, np.float64),
                        velocities=np.asarray(velocities, np.float64),
                        **{k: np.asarray(v) for k, v in extra.items()})


def load_state(path):
    """(positions, velocities, extra dict) saved by save_state."""
    with np.load(path) as z:
        extra = {k: z[k] for k in z.files if k not in ("positions", "velocities")}
        return z["positions"], z["velocities"], extra
