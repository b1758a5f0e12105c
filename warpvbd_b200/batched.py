"""Many independent VBD environments stepped in one launch.

The reference batches environments by concatenating their meshes into one
``VBDSolver`` (mmichelis/WarpVBD examples/run_mass_spring_parallel.py:35-58):
one colouring, one global convergence test, so every environment runs as many
sweeps as the slowest.  Here the environments keep their own convergence test
and sweep count: block mode gives each environment one thread block that runs
its whole step (all sweeps and colours) with the environment's displacements
in shared memory.
"""
import ctypes

import numpy as np

from . import _lib
from .vbd_solver import (_device_index, _host, _host_out, _set_warmstart, _ws_features,
                         _ws_targets)


class BatchedVBDSolver:
    """``envs``: sequence of objects with ``vertices``, ``tets``, ``density``,
    ``youngs``, ``poisson``, ``active`` (warpvbd_b200.scenes.Scene) or dicts
    with the ``VBDSolver`` argument names."""

    def __init__(self, envs, damping_coefficient=0.0, gravity=(0.0, 0.0, -9.81), dx_tol=1e-7,
                 max_iter=1000, device="cuda", *, material="snh", precision="fp64",
                 tpv=0, block_threads=0, cluster=0, order_index=False, tiered=False,
                 wide_tier=None, tune=False, gpu_setup=False):
        """``cluster``: blocks per thread-block cluster (0 = automatic); an
        environment much heavier than the others runs on a whole cluster.
        ``tiered``: run the environments split over a cluster in one launch
        and all others, one block each with shared memory sized for the
        largest of them, in a second launch beside it.
        ``wide_tier`` (with ``tiered``; None = on): a third launch with
        clusters twice that size for the environments the planner predicts
        would otherwise set the step time (it is used only on steps where
        the duration model says it helps; results are bit-identical).
        ``tune``: pick tpv / block_threads / cluster / order_index / tiered
        with the autotuner (warpvbd_b200.autotune; measured once, then
        cached).  ``gpu_setup``: colour all environments in one GPU pass
        (the same colours as the host's per-environment pass)."""
        if tune:
            from . import autotune
            cfg = autotune.tune_batched(envs, material=material, precision=precision,
                                        device=device, dx_tol=dx_tol, max_iter=max_iter)
            tpv, block_threads = cfg["tpv"], cfg["block_threads"]
            cluster, order_index = cfg["cluster"], cfg["order_index"]
            tiered = cfg.get("tiered", False)
            wide_tier = cfg.get("wide_tier", wide_tier)
        self.device = device
        Xs, Ts, rho, E, nu, act = [], [], [], [], [], []
        voff, toff = [0], [0]
        for env in envs:
            get = (lambda k, a: env[k]) if isinstance(env, dict) else (lambda k, a: getattr(env, a))
            X = np.asarray(_host(get("initial_positions", "vertices")), np.float64).reshape(-1, 3)
            t = np.asarray(_host(get("elements", "tets")), np.int64).reshape(-1, 4)
            Xs.append(X)
            Ts.append(t + voff[-1])
            rho.append(np.asarray(_host(get("densities", "density")), np.float64))
            E.append(np.asarray(_host(get("youngs_modulus", "youngs")), np.float64))
            nu.append(np.asarray(_host(get("poissons_ratio", "poisson")), np.float64))
            a = get("active_mask", "active")
            act.append(np.ones(X.shape[0], bool) if a is None else np.asarray(_host(a), bool))
            voff.append(voff[-1] + X.shape[0])
            toff.append(toff[-1] + t.shape[0])
        self.n_env = len(Xs)
        self.env_vertex_offset = np.asarray(voff, np.int32)
        self.env_tet_offset = np.asarray(toff, np.int32)
        X = _lib.f64(np.concatenate(Xs))
        tets = _lib.i32(np.concatenate(Ts))
        rho, E, nu = (_lib.f64(np.concatenate(a)) for a in (rho, E, nu))
        actu8 = np.ascontiguousarray(np.concatenate(act).astype(np.uint8))
        g = _lib.f64(gravity, (3,))
        flags = {"snh": _lib.MATERIAL_SNH, "stvk": _lib.MATERIAL_STVK}[material]
        flags |= _lib.PRECISIONS[precision]
        flags |= _lib.MODE_BLOCK
        flags |= _lib.cluster_flags(cluster)
        if order_index:
            flags |= _lib.ORDER_INDEX
        if tiered:
            flags |= _lib.TIERED
            if wide_tier is None or wide_tier:
                flags |= _lib.TIERED_WIDE
        if gpu_setup:
            flags |= _lib.GPU_SETUP
        L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(L.vbd_create_batched(
            _lib.ptr(X, "d"), X.shape[0], _lib.ptr(tets, "i"), tets.shape[0], _lib.ptr(rho, "d"),
            _lib.ptr(E, "d"), _lib.ptr(nu, "d"), actu8.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            float(damping_coefficient), _lib.ptr(g, "d"), _lib.ptr(self.env_vertex_offset, "i"),
            _lib.ptr(self.env_tet_offset, "i"), self.n_env, flags, int(tpv), int(block_threads),
            _device_index(device), ctypes.byref(h)), "vbd_create_batched")
        self._h = h
        self.n_vertices = X.shape[0]
        self.initial_positions = X.copy()
        self.dx_tol = dx_tol
        self.max_iter = max_iter
        self.last_iterations = np.zeros(self.n_env, np.int32)
        self.last_status = _lib.OK

    def info(self):
        inf = _lib.VBDInfo()
        _lib.check(_lib.load().vbd_get_info(self._h, ctypes.byref(inf)))
        return {n: getattr(inf, n) for n, _ in _lib.VBDInfo._fields_}

    @property
    def stream(self):
        return _lib.load().vbd_get_stream(self._h)

    def set_trace(self, enable=True):
        """Record a timeline of every later step (block mode): per thread
        block of the environment launches, its start and end on the GPU's
        global timer; see ``timeline``."""
        _lib.check(_lib.load().vbd_set_trace(self._h, 1 if enable else 0), "vbd_set_trace")

    def timeline(self):
        """Timeline of the last finished traced step, one row per thread
        block: dict of arrays start_ns, end_ns (relative to the earliest
        start), env, rank (in its cluster), sm, sweeps, launch (0 the single
        or split launch, 1 the light launch of a tiered step, 2 its wide
        tier)."""
        L = _lib.load()
        n = ctypes.c_int(0)
        _lib.check(L.vbd_get_trace(self._h, None, 0, ctypes.byref(n)), "vbd_get_trace")
        cap = n.value
        rec = np.zeros((max(cap, 1), 4), np.uint64)
        _lib.check(L.vbd_get_trace(self._h, rec.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)),
                                   cap, ctypes.byref(n)), "vbd_get_trace")
        rec = rec[:n.value]
        rec = rec[rec[:, 0] > 0]  # padding blocks of a cluster record nothing
        t0 = rec[:, 0].min() if len(rec) else np.uint64(0)
        return {"start_ns": (rec[:, 0] - t0).astype(np.int64),
                "end_ns": (rec[:, 1] - t0).astype(np.int64),
                "env": (rec[:, 2] >> np.uint64(32)).astype(np.int64),
                "rank": ((rec[:, 2] >> np.uint64(16)) & np.uint64(0xFFFF)).astype(np.int64),
                "sm": (rec[:, 2] & np.uint64(0xFFFF)).astype(np.int64),
                "sweeps": (rec[:, 3] >> np.uint64(8)).astype(np.int64),
                "launch": (rec[:, 3] & np.uint64(0xFF)).astype(np.int64)}

    def step(self, dt=1e-3, dx_tol=None, tol_per_env=None, max_iter=None, blocking=True,
             out=None):
        """Step every environment; returns the per-environment sweep counts
        (blocking) or None (enqueued only; see ``sync``).  ``out``: a
        C-contiguous float64 [n_vertices, 3] array that receives the new
        positions (blocking); page-locked memory (e.g. a torch tensor made
        with pin_memory=True) is written by the step kernels themselves as
        each environment finishes."""
        L = _lib.load()
        tol = self.dx_tol if dx_tol is None else dx_tol
        mi = self.max_iter if max_iter is None else max_iter
        tpe = None if tol_per_env is None else _lib.f64(tol_per_env, (self.n_env,))
        if out is not None:
            out = _host_out(out, self.n_vertices)
            it = np.zeros(self.n_env, np.int32)
            st = L.vbd_step_batched_to(self._h, float(dt), float(tol), _lib.ptr(tpe, "d"), int(mi),
                                       it.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                       _lib.ptr(out, "d"))
            self._after(st, it)
            return it
        if blocking:
            it = np.zeros(self.n_env, np.int32)
            st = L.vbd_step_batched(self._h, float(dt), float(tol), _lib.ptr(tpe, "d"), int(mi),
                                    it.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
            self._after(st, it)
            return it
        _lib.check(L.vbd_step_batched(self._h, float(dt), float(tol), _lib.ptr(tpe, "d"),
                                      int(mi), None), "vbd_step_batched")
        return None

    def sync(self):
        L = _lib.load()
        st = L.vbd_sync(self._h)
        it = np.zeros(self.n_env, np.int32)
        L.vbd_get_iterations(self._h, it.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        self._after(st, it)
        return it

    def _after(self, st, it):
        self.last_status = st
        self.last_iterations = it
        if st == _lib.ERR_NONFINITE:
            raise FloatingPointError("VBD step produced non-finite positions")
        _lib.check(st, "vbd_step_batched")

    def positions(self, out=None):
        """float64 [V, 3]; `out`: an existing C-contiguous float64 array to fill
        (e.g. page-locked, for fast transfers)."""
        out = _host_out(out, self.n_vertices)
        _lib.check(_lib.load().vbd_get_positions(self._h, _lib.ptr(out, "d")))
        return out

    def velocities(self, out=None):
        out = _host_out(out, self.n_vertices)
        _lib.check(_lib.load().vbd_get_velocities(self._h, _lib.ptr(out, "d")))
        return out

    def env_slice(self, e):
        return slice(int(self.env_vertex_offset[e]), int(self.env_vertex_offset[e + 1]))

    def set_state(self, positions=None, velocities=None):
        L = _lib.load()
        if positions is not None:
            x = _lib.f64(positions, (self.n_vertices, 3))
            _lib.check(L.vbd_set_positions(self._h, _lib.ptr(x, "d")))
        if velocities is not None:
            v = _lib.f64(velocities, (self.n_vertices, 3))
            _lib.check(L.vbd_set_velocities(self._h, _lib.ptr(v, "d")))

    def reset(self):
        _lib.check(_lib.load().vbd_reset(self._h))

    # ---- learned warm start (see warpvbd_b200.warmstart) --------------------
    def set_warmstart(self, params):
        return _set_warmstart(self._h, params)

    def ws_features(self, dt, out=None):
        return _ws_features(self._h, self.n_vertices, dt, out)

    def incremental_potential(self, positions, dt=1e-3):
        """Per-environment incremental potential at `positions` (caller order)
        for a step of length dt from the current state: the strain energy of
        every tet with a solved vertex plus the solved vertices' inertia
        energy, as the learned warm start's check evaluates it."""
        x = _lib.f64(positions, (self.n_vertices, 3))
        out = np.zeros(self.n_env)
        _lib.check(_lib.load().vbd_incremental_potential(self._h, float(dt), _lib.ptr(x, "d"),
                                                         _lib.ptr(out, "d")),
                   "vbd_incremental_potential")
        return out

    def ws_vertex_rows(self):
        """Row of every vertex (caller order) in the feature, target and
        prediction arrays."""
        rows = np.zeros(self.n_vertices, np.int32)
        _lib.check(_lib.load().vbd_ws_vertex_rows(self._h, _lib.ptr(rows, "i")),
                   "vbd_ws_vertex_rows")
        return rows

    def ws_targets(self, features, out=None):
        return _ws_targets(self._h, self.n_vertices, features, out)

    def ws_predict(self, features, out=None):
        import torch
        if out is None:
            out = torch.empty((self.n_vertices, 4), device=features.device)
        _lib.check(_lib.load().vbd_ws_predict(self._h, ctypes.c_void_p(features.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr())), "vbd_ws_predict")
        return out

    def env_status(self):
        """Per-environment status bits of the last step (16 = warm start used)."""
        out = np.zeros(self.n_env, np.uint32)
        _lib.check(_lib.load().vbd_get_env_status(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))))
        return out

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
