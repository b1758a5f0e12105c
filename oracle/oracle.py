"""ctypes front end of the FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle_vbd.so`` (built from ``vbd_oracle.c`` by
``make -C oracle``), the CPU restatement of the reference solver
(mmichelis/WarpVBD src/vbd_solver.py:15-612, src/coloring.py:24-72).  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this module; the product package never does.

``OracleSolver`` mirrors ``VBDSolver`` (vbd_solver.py:366-612): construct with
the mesh and material arrays, then ``step(positions, dt, dx_tol)``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_vbd.so")
_lib = None

SNH, STVK = 0, 1

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)


def build():
    """Compile the oracle library in place (gcc + OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, _d, ctypes.c_int, _i, _d, _d, _d, _u8,
                                 ctypes.c_double, _d, ctypes.c_int, ctypes.c_int, _i]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_step.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.c_void_p, _d, ctypes.c_double, ctypes.c_double,
                               ctypes.c_int, _d, ctypes.POINTER(ctypes.c_int)]
        L.orc_reset.argtypes = [ctypes.c_void_p]
        for name in ("orc_num_colors", "orc_max_group", "orc_max_incident", "orc_bad_dm"):
            getattr(L, name).restype = ctypes.c_int
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.orc_guard_hits.restype = ctypes.c_longlong
        L.orc_guard_hits.argtypes = [ctypes.c_void_p]
        L.orc_color_table.argtypes = [ctypes.c_void_p, _i]
        L.orc_adjacency.argtypes = [ctypes.c_void_p, _i]
        L.orc_element_data.argtypes = [ctypes.c_void_p, _d, _d, _d, _d, _d]
        L.orc_get_state.argtypes = [ctypes.c_void_p, _d, _d]
        L.orc_set_state.argtypes = [ctypes.c_void_p, _d, _d]
        L.orc_vertex_grad_hess.argtypes = [ctypes.c_void_p, ctypes.c_int, _d, ctypes.c_double,
                                           _d, _d]
        L.orc_incremental_potential.restype = ctypes.c_double
        L.orc_incremental_potential.argtypes = [ctypes.c_void_p, _d, ctypes.c_double]
        L.orc_tet_grad_hess.argtypes = [ctypes.c_int, _d, _d, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, _d, _d]
        L.orc_tet_energy.restype = ctypes.c_double
        L.orc_tet_energy.argtypes = [ctypes.c_int, _d, _d, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double]
        L.orc_graph_coloring.restype = ctypes.c_int
        L.orc_graph_coloring.argtypes = [ctypes.c_int, _i, _i, ctypes.POINTER(ctypes.c_int)]
        L.orc_lame.argtypes = [ctypes.c_int, _d, _d, _d, _d]
        L.orc_invdm_mass_volume.restype = ctypes.c_int
        L.orc_invdm_mass_volume.argtypes = [_d, ctypes.c_int, _i, _d, _d, _d, _d]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(shape) if shape is not None else a


def set_threads(n):
    lib().orc_set_threads(int(n))


def max_threads():
    return lib().orc_max_threads()


def graph_coloring(tets):
    """coloring.py:24-72 restated: greedy colour per vertex (len max(tets)+1)."""
    tets = np.ascontiguousarray(np.asarray(tets, dtype=np.int32))
    nv = int(tets.max()) + 1 if tets.size else 0
    out = np.empty(max(nv, 1), dtype=np.int32)
    n = ctypes.c_int(0)
    ncol = lib().orc_graph_coloring(tets.shape[0], _p(tets, _i), _p(out, _i), ctypes.byref(n))
    if ncol < 0:
        raise AssertionError("Exceeded maximum number of colors")
    return out[:n.value]


def tet_grad_hess(material, x4, inv_dm, mu, lam, vol, a):
    x4 = _f64(x4, (12,))
    inv_dm = _f64(inv_dm, (9,))
    g = np.zeros(3)
    h = np.zeros(9)
    lib().orc_tet_grad_hess(material, _p(x4, _d), _p(inv_dm, _d), mu, lam, vol, a,
                            _p(g, _d), _p(h, _d))
    return g, h.reshape(3, 3)


def tet_energy(material, x4, inv_dm, mu, lam, vol):
    x4 = _f64(x4, (12,))
    inv_dm = _f64(inv_dm, (9,))
    return lib().orc_tet_energy(material, _p(x4, _d), _p(inv_dm, _d), mu, lam, vol)


class OracleSolver:
    """FP64 restatement of VBDSolver (vbd_solver.py:366-612).

    ``guarded=False`` reproduces the reference exactly (a non-positive-definite
    3x3 block gives NaN); ``guarded=True`` applies the product's guarded
    Newton step (inertia-only Hessian fallback)."""

    def __init__(self, initial_positions, elements, densities, youngs_modulus, poissons_ratio,
                 damping_coefficient=1.0, active_mask=None, gravity=(0.0, 0.0, -9.81),
                 dx_tol=1e-9, max_iter=100, material="snh", guarded=False, coloring=None):
        L = lib()
        X = _f64(initial_positions)
        self.V = X.shape[0]
        tets = np.ascontiguousarray(np.asarray(elements, dtype=np.int32))
        self.T = tets.shape[0]
        rho = _f64(densities)
        E = _f64(youngs_modulus)
        nu = _f64(poissons_ratio)
        act = None if active_mask is None else np.ascontiguousarray(
            np.asarray(active_mask, dtype=np.uint8))
        g = _f64(gravity)
        col = None if coloring is None else np.ascontiguousarray(np.asarray(coloring, np.int32))
        mat = {"snh": SNH, "stvk": STVK}[material]
        self._h = L.orc_create(self.V, _p(X, _d), self.T, _p(tets, _i), _p(rho, _d), _p(E, _d),
                               _p(nu, _d), _p(act, _u8), float(damping_coefficient), _p(g, _d),
                               mat, int(bool(guarded)), _p(col, _i))
        self.initial_positions = X.copy()
        self.dx_tol = dx_tol
        self.max_iter = max_iter
        self.last_iterations = 0
        self.warned = False

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    @property
    def old_positions(self):
        x = np.empty((self.V, 3))
        lib().orc_get_state(self._h, _p(x, _d), None)
        return x

    @property
    def old_velocities(self):
        v = np.empty((self.V, 3))
        lib().orc_get_state(self._h, None, _p(v, _d))
        return v

    def set_state(self, x=None, v=None):
        x = None if x is None else _f64(x, (self.V, 3))
        v = None if v is None else _f64(v, (self.V, 3))
        lib().orc_set_state(self._h, _p(x, _d), _p(v, _d))

    @property
    def color_groups(self):
        L = lib()
        nc, mg = L.orc_num_colors(self._h), L.orc_max_group(self._h)
        out = np.empty((nc, mg), dtype=np.int32)
        L.orc_color_table(self._h, _p(out, _i))
        return out

    @property
    def adj_v2e(self):
        L = lib()
        K = L.orc_max_incident(self._h)
        out = np.empty((self.V, K), dtype=np.int32)
        L.orc_adjacency(self._h, _p(out, _i))
        return out

    def element_data(self):
        T = self.T
        inv = np.empty((T, 3, 3))
        m, v, mu, lam = (np.empty(T) for _ in range(4))
        lib().orc_element_data(self._h, _p(inv, _d), _p(m, _d), _p(v, _d), _p(mu, _d),
                               _p(lam, _d))
        return {"inv_Dm": inv, "masses": m, "volumes": v, "lame_mus": mu, "lame_lambdas": lam}

    @property
    def bad_dm(self):
        return lib().orc_bad_dm(self._h)

    @property
    def guard_hits(self):
        return lib().orc_guard_hits(self._h)

    def reset(self):
        lib().orc_reset(self._h)

    def step(self, positions=None, dt=1e-3, dx_tol=None, max_iter=None):
        tol = self.dx_tol if dx_tol is None else dx_tol
        mi = self.max_iter if max_iter is None else max_iter
        pos = None if positions is None else _f64(positions, (self.V, 3))
        out = np.empty((self.V, 3))
        it = ctypes.c_int(0)
        self.warned = bool(lib().orc_step(self._h, _p(pos, _d), float(dt), float(tol), int(mi),
                                          _p(out, _d), ctypes.byref(it)))
        self.last_iterations = it.value
        return out

    def vertex_grad_hess(self, v, x, dt):
        x = _f64(x, (self.V, 3))
        g = np.zeros(3)
        h = np.zeros(9)
        lib().orc_vertex_grad_hess(self._h, int(v), _p(x, _d), float(dt), _p(g, _d), _p(h, _d))
        return g, h.reshape(3, 3)

    def incremental_potential(self, x, dt):
        x = _f64(x, (self.V, 3))
        return lib().orc_incremental_potential(self._h, _p(x, _d), float(dt))
