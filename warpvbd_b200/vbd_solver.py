"""Drop-in ``VBDSolver`` backed by the sm_100a CUDA solver in libvbd_b200.so.

Mirrors the reference's interface (mmichelis/WarpVBD src/vbd_solver.py:366-612):
the constructor takes the tet mesh, per-tet density / Young's modulus /
Poisson's ratio, damping, an active mask, gravity, ``dx_tol`` and
``max_iter``; ``step(positions, dt, dx_tol=None)`` advances one implicit-Euler
step and returns the new positions; ``reset()`` restores the initial state.
Callers use it exactly like the reference::

    solver = VBDSolver(X, tets, rho, E, nu, damping_coefficient=0.0,
                       active_mask=mask, dx_tol=1e-7, max_iter=1000)
    for _ in range(300):
        x = solver.step(solver.old_positions, 1e-3)
        tip = x.numpy()[tip_idx].mean(axis=0)

Arrays may be numpy arrays, torch tensors or any object with ``.numpy()``.
The solver state stays on the GPU; ``step`` returns a ``DeviceArray`` view
whose ``.numpy()`` copies the positions to the host.  As with the reference's
drivers, read a returned array before the following ``step``: a view of an
overwritten state raises instead of returning stale data (``copy()`` keeps
a host snapshot).
"""
import ctypes

import numpy as np

from . import _lib
from .coloring import color_groups_table

EPS = 1e-12                     # vbd_solver.py:11
MAX_ELEMENTS_PER_VERTEX = 32    # vbd_solver.py:12


def _host(a, dtype=None):
    """numpy view of a numpy / torch / Warp-like array."""
    if a is None:
        return None
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    elif not isinstance(a, np.ndarray) and hasattr(a, "numpy"):
        a = a.numpy()
    a = np.asarray(a)
    return a.astype(dtype, copy=False) if dtype is not None else a


def _device_index(device):
    if device is None:
        return 0
    if isinstance(device, int):
        return device
    d = str(device)
    if d.startswith("cuda"):
        return int(d.split(":")[1]) if ":" in d else 0
    raise ValueError(f"warpvbd_b200 runs on CUDA devices only (got device={device!r}); "
                     "there is no CPU path")


def _host_out(out, n):
    """A float64 [n, 3] C-contiguous host array to download into."""
    if out is None:
        return np.empty((n, 3))
    if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (n, 3)
            or not out.flags.c_contiguous):
        raise ValueError(f"out must be a C-contiguous float64 array of shape ({n}, 3)")
    return out


def _set_warmstart(handle, model):
    """Enable the learned warm start, or disable it (None).  `model` is a
    (params, norm) pair as returned by warmstart.load / train_warmstart, or
    bare parameters (identity normalisation)."""
    L = _lib.load()
    if model is None:
        return _lib.check(L.vbd_set_warmstart(handle, None, None), "vbd_set_warmstart")
    params, norm = model if isinstance(model, tuple) else (model, None)
    fp = ctypes.POINTER(ctypes.c_float)
    p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(-1))
    if p.size != L.vbd_ws_param_count():
        raise ValueError(f"expected {L.vbd_ws_param_count()} parameters, got {p.size}")
    n = None if norm is None else np.ascontiguousarray(np.asarray(norm, np.float32).reshape(-1))
    if n is not None and n.size != 50:
        raise ValueError("the normalisation vector holds 50 values")
    return _lib.check(L.vbd_set_warmstart(handle, p.ctypes.data_as(fp),
                                          None if n is None else n.ctypes.data_as(fp)),
                      "vbd_set_warmstart")


def _ws_features(handle, n, dt, out):
    import torch
    L = _lib.load()
    if out is None:
        out = torch.empty((n, L.vbd_ws_feature_width()), device="cuda")
    _lib.check(L.vbd_ws_features(handle, float(dt), ctypes.c_void_p(out.data_ptr())),
               "vbd_ws_features")
    return out


def _ws_targets(handle, n, features, out):
    import torch
    if out is None:
        out = torch.empty((n, 3), device=features.device)
    _lib.check(_lib.load().vbd_ws_targets(handle, ctypes.c_void_p(features.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr())), "vbd_ws_targets")
    return out


class DeviceArray:
    """A vertex array (positions or velocities) held on the GPU by a solver.

    ``numpy()`` returns a float64 [V, 3] host copy in the caller's vertex
    order.  The view is tied to one solver state version."""

    def __init__(self, solver, version, kind):
        self._solver = solver
        self._version = version
        self._kind = kind
        self._host = None

    @property
    def shape(self):
        return (self._solver.n_vertices, 3)

    def __len__(self):
        return self._solver.n_vertices

    def numpy(self, out=None):
        """Host copy (float64 [V, 3]); `out`: an existing C-contiguous float64
        array to fill instead (e.g. page-locked, for fast transfers)."""
        if self._host is not None:
            if out is None:
                return self._host.copy()
            out[...] = self._host
            return out
        if self._version != self._solver._version:
            raise RuntimeError(
                "this array's solver state was overwritten by a later step or reset; call "
                ".numpy() (or .copy()) before stepping again")
        return self._solver._download(self._kind, out)

    def copy(self):
        """Materialise a host snapshot that survives later steps."""
        if self._host is None:
            self._host = self.numpy()
        return self

    def __array__(self, dtype=None, copy=None):
        a = self.numpy()
        return a.astype(dtype) if dtype is not None else a


class VBDSolver:
    """Vertex Block Descent solver on one GPU (reference: vbd_solver.py:366).

    Extra keyword arguments (all optional, not in the reference):
      material   "snh" (Stable Neo-Hookean, the reference's active model) or
                 "stvk" (St. Venant-Kirchhoff, the reference's commented model)
      precision  "fp64" (default: state and arithmetic in double precision, as in
                 the reference, whose types are all float64), "mixed" (fp64
                 positions and velocities, fp32 per-slot arithmetic: faster, but
                 fp32 rounding moves the stopping sweep of some steps, so long
                 trajectories drift from the fp64 one; measured up to 1.6e-5 of
                 the bounding-box diagonal on the 160x16x16 cantilever over 300
                 steps and 9.6e-5 on the 256-environment batch) or "fp32"
                 (everything fp32)
      mode       "auto", "block", "graph", "hostloop" or "persist" (see include/vbd_b200.h)
      tpv, block_threads   launch shape (0 = automatic)
      cluster    block mode: spread the mesh over this many thread blocks of one
                 cluster (1 to 16; 0 = automatic)
      order_index  keep ascending vertex index inside a colour (default: by valence)
      tune       pick mode / tpv / block_threads / cluster / order_index with the
                 autotuner (warpvbd_b200.autotune; measured once per mesh and GPU
                 type, then cached)
      coloring   per-vertex colours to use instead of the greedy colouring
      strict_spd raise instead of taking the guarded step on a non-SPD block
      gpu_setup  colour the mesh on the GPU at construction (the same colours as
                 the host pass; vbd_graph_coloring_gpu)
      persist_sync  persistent mode: "neighbours" (default; each block waits
                 between colours only for the blocks whose vertices share a
                 tet with its own) or "grid" (a grid barrier between colours)
      allow_high_valence  lift the reference's 32 incident-tets limit
    """

    def __init__(self, initial_positions, elements, densities, youngs_modulus, poissons_ratio,
                 damping_coefficient=1.0, active_mask=None, gravity=(0.0, 0.0, -9.81),
                 dx_tol=1e-9, max_iter=100, device="cuda", *, material="snh",
                 precision="fp64", mode="auto", tpv=0, block_threads=0, cluster=0, coloring=None,
                 strict_spd=False, allow_high_valence=False, verbose=False, order_index=False,
                 tune=False, persist_sync="neighbours", gpu_setup=False):
        L = _lib.load()
        if tune:
            from . import autotune
            cfg = autotune.tune_single(
                dict(initial_positions=_host(initial_positions), elements=_host(elements),
                     densities=_host(densities), youngs_modulus=_host(youngs_modulus),
                     poissons_ratio=_host(poissons_ratio),
                     active_mask=None if active_mask is None else _host(active_mask)),
                material=material, precision=precision, device=device,
                damping_coefficient=damping_coefficient)
            mode, tpv, block_threads = cfg["mode"], cfg["tpv"], cfg["block_threads"]
            cluster, order_index = cfg["cluster"], cfg["order_index"]
        X = _lib.f64(_host(initial_positions), (-1, 3))
        tets = _lib.i32(_host(elements)).reshape(-1, 4)
        rho = _lib.f64(_host(densities))
        E = _lib.f64(_host(youngs_modulus))
        nu = _lib.f64(_host(poissons_ratio))
        act = None if active_mask is None else np.ascontiguousarray(
            _host(active_mask).astype(np.uint8))
        g = _lib.f64(_host(gravity), (3,))
        col = None if coloring is None else _lib.i32(_host(coloring))
        self.n_vertices = X.shape[0]
        self.n_elements = tets.shape[0]
        for name, arr in (("densities", rho), ("youngs_modulus", E), ("poissons_ratio", nu)):
            if arr.shape != (self.n_elements,):
                raise ValueError(f"{name} must hold one value per element")
        if act is not None and act.shape != (self.n_vertices,):
            raise ValueError("active_mask must hold one value per vertex")
        flags = {"snh": _lib.MATERIAL_SNH, "stvk": _lib.MATERIAL_STVK}[material]
        flags |= _lib.PRECISIONS[precision]
        flags |= _lib.MODES[mode]
        if strict_spd:
            flags |= _lib.STRICT_SPD
        if order_index:
            flags |= _lib.ORDER_INDEX
        if persist_sync not in ("neighbours", "grid"):
            raise ValueError('persist_sync must be "neighbours" or "grid"')
        if persist_sync == "grid":
            flags |= _lib.PERSIST_GRID_BARRIERS
        if gpu_setup:
            flags |= _lib.GPU_SETUP
        flags |= _lib.cluster_flags(cluster)
        self.device = device
        self._dev = _device_index(device)
        h = ctypes.c_void_p()
        _lib.check(L.vbd_create(_lib.ptr(X, "d"), X.shape[0], _lib.ptr(tets, "i"),
                                tets.shape[0], _lib.ptr(rho, "d"), _lib.ptr(E, "d"),
                                _lib.ptr(nu, "d"), _lib.ptr(act, "u8"),
                                float(damping_coefficient), _lib.ptr(g, "d"),
                                _lib.ptr(col, "i"), flags, int(tpv), int(block_threads),
                                self._dev, ctypes.byref(h)), "vbd_create")
        self._h = h
        self._version = 0
        self.initial_positions = X.copy()
        self.elements = tets
        self.densities = rho
        self.youngs_modulus = E
        self.poissons_ratio = nu
        self.damping_coefficient = float(damping_coefficient)
        self.active_mask = (np.ones(self.n_vertices, dtype=bool) if act is None
                            else act.astype(bool))
        self.gravity = g
        self.dx_tol = dx_tol
        self.max_iter = max_iter
        self.material = material
        self.precision = precision
        self.allow_high_valence = allow_high_valence
        self.last_iterations = 0
        self.last_status = _lib.OK
        self.old_positions = DeviceArray(self, self._version, "x")
        info = self.info()
        self.max_incident_elements = info["max_valence"]
        if verbose:
            print(f"Assigned {info['n_colors']} colors. Max incident elements per vertex: "
                  f"{self.max_incident_elements}")

    # ---- reference attributes ---------------------------------------------
    @property
    def old_velocities(self):
        return DeviceArray(self, self._version, "v")

    @property
    def color_groups(self):
        """int32 [n_colors, max_group] of vertex ids, -1 padded (vbd_solver.py:476-483)."""
        L = _lib.load()
        nc, mg = ctypes.c_int(0), ctypes.c_int(0)
        _lib.check(L.vbd_get_color_groups(self._h, None, ctypes.byref(nc), ctypes.byref(mg)))
        out = np.full((nc.value, mg.value), -1, dtype=np.int32)
        if out.size:
            _lib.check(L.vbd_get_color_groups(self._h, _lib.ptr(out, "i"), None, None))
        return out

    @property
    def adj_v2e(self):
        """int32 [V, max_incident] incident tets, ascending, -1 padded (vbd_solver.py:485-498)."""
        V, K = self.n_vertices, self.max_incident_elements
        out = np.full((V, K), -1, dtype=np.int32)
        flat = self.elements.reshape(-1)
        tet_of = np.repeat(np.arange(self.n_elements, dtype=np.int32), 4)
        order = np.lexsort((tet_of, flat))
        v_sorted, t_sorted = flat[order], tet_of[order]
        starts = np.searchsorted(v_sorted, np.arange(V))
        pos = np.arange(v_sorted.size) - starts[v_sorted]
        out[v_sorted, pos] = t_sorted
        return out

    def lame_parameters(self):
        """(mu, lambda) per tet (convert_youngs_poisson_to_lame, vbd_solver.py:345-362)."""
        E, nu = self.youngs_modulus, self.poissons_ratio
        return E / (2.0 * (1.0 + nu)), (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def incremental_potential(self, positions, dt=1e-3):
        """Incremental potential at `positions` for a step of length dt from
        the current state (strain energy of the tets with a solved vertex plus
        the solved vertices' inertia energy; no counterpart in the reference,
        whose step descends its gradient)."""
        x = _lib.f64(positions, (self.n_vertices, 3))
        out = np.zeros(1)
        _lib.check(_lib.load().vbd_incremental_potential(self._h, float(dt), _lib.ptr(x, "d"),
                                                         _lib.ptr(out, "d")),
                   "vbd_incremental_potential")
        return float(out[0])

    def info(self):
        L = _lib.load()
        inf = _lib.VBDInfo()
        _lib.check(L.vbd_get_info(self._h, ctypes.byref(inf)))
        return {n: getattr(inf, n) for n, _ in _lib.VBDInfo._fields_}

    @property
    def stream(self):
        return _lib.load().vbd_get_stream(self._h)

    # ---- state --------------------------------------------------------------
    def _download(self, kind, out=None):
        L = _lib.load()
        out = _host_out(out, self.n_vertices)
        fn = L.vbd_get_positions if kind == "x" else L.vbd_get_velocities
        _lib.check(fn(self._h, _lib.ptr(out, "d")), "download")
        return out

    def set_state(self, positions=None, velocities=None):
        """Overwrite the current positions and / or velocities (float64 [V, 3])."""
        L = _lib.load()
        if positions is not None:
            x = _lib.f64(_host(positions), (self.n_vertices, 3))
            _lib.check(L.vbd_set_positions(self._h, _lib.ptr(x, "d")), "set_positions")
        if velocities is not None:
            v = _lib.f64(_host(velocities), (self.n_vertices, 3))
            _lib.check(L.vbd_set_velocities(self._h, _lib.ptr(v, "d")), "set_velocities")
        self._bump()

    def get_state(self):
        return self._download("x"), self._download("v")

    def _bump(self):
        self._version += 1
        self.old_positions = DeviceArray(self, self._version, "x")

    def reset(self):
        """Positions back to the initial positions, velocities to zero (vbd_solver.py:501-506)."""
        _lib.check(_lib.load().vbd_reset(self._h), "vbd_reset")
        self._bump()

    def step(self, positions=None, dt=1e-3, dx_tol=None, *, max_iter=None, blocking=True):
        """One time step from ``positions`` (vbd_solver.py:509-612); returns the new positions.

        ``positions`` is normally ``solver.old_positions`` (as every reference
        driver passes); any other array is uploaded first.  With
        ``blocking=False`` the step is only enqueued on the solver's stream and
        ``last_iterations`` is updated by ``sync()``."""
        if (MAX_ELEMENTS_PER_VERTEX < self.max_incident_elements
                and not self.allow_high_valence):
            raise AssertionError(
                "MAX_ELEMENTS_PER_VERTEX is smaller than the maximum number of incident "
                "elements per vertex. Increase this constant and recompile.")
        tol = self.dx_tol if dx_tol is None else dx_tol
        mi = self.max_iter if max_iter is None else max_iter
        if positions is not None and positions is not self.old_positions:
            if isinstance(positions, DeviceArray) and positions._solver is self \
                    and positions._version == self._version:
                pass
            else:
                self.set_state(positions=positions)
        L = _lib.load()
        if blocking:
            it = ctypes.c_int(0)
            st = L.vbd_step(self._h, float(dt), float(tol), int(mi), ctypes.byref(it))
            self._after_step(st, it.value, mi)
        else:
            _lib.check(L.vbd_step(self._h, float(dt), float(tol), int(mi), None), "vbd_step")
            self._pending_max_iter = mi
        self._bump()
        return self.old_positions

    def sync(self):
        L = _lib.load()
        st = L.vbd_sync(self._h)
        it = ctypes.c_int(0)
        L.vbd_get_iterations(self._h, ctypes.byref(it))
        self._after_step(st, it.value, getattr(self, "_pending_max_iter", self.max_iter))
        return self.last_iterations

    def _after_step(self, status, iterations, max_iter):
        self.last_status = status
        self.last_iterations = iterations
        if status == _lib.ERR_NONFINITE:
            raise FloatingPointError(
                "VBD step produced non-finite positions: "
                + _lib.load().vbd_last_error_message().decode(errors="replace"))
        _lib.check(status, "vbd_step")
        if iterations == max_iter:   # the reference's warning condition (vbd_solver.py:581-582)
            dx = np.full(1, np.nan)
            _lib.load().vbd_get_final_dx(self._h, _lib.ptr(dx, "d"))
            print("Warning: VBD solver did not converge within the maximum number of "
                  f"iterations. Final dx max: {float(dx[0])}")

    # ---- learned warm start (see warpvbd_b200.warmstart) --------------------
    def set_warmstart(self, params):
        """Start every step from the network's prediction when it lowers the
        incremental potential (params: fp32 array, None disables)."""
        return _set_warmstart(self._h, params)

    def ws_features(self, dt, out=None):
        return _ws_features(self._h, self.n_vertices, dt, out)

    def ws_targets(self, features, out=None):
        return _ws_targets(self._h, self.n_vertices, features, out)

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.load().vbd_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["VBDSolver", "DeviceArray", "EPS", "MAX_ELEMENTS_PER_VERTEX", "color_groups_table"]
