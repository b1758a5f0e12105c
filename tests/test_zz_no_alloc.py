"""vbd_step_noalloc against vbd_step (GPU, through the C ABI).

vbd_step_noalloc serves callers that may not allocate GPU memory once they
are stepping (an application that commits its device-memory budget at
start-up, a real-time loop whose per-step code may not call an allocator):
it keeps the sweep's scratch in a static device array instead of allocating.
Two solvers are built from the same mesh; one is stepped with vbd_step
(graph mode), the other with vbd_step_noalloc, twice in a row, and their
positions must agree within the tolerance of the other GPU parity tests
(1e-5 of the bounding-box diagonal), with the same sweep counts.  The file
is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from warpvbd_b200 import _lib, scenes

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5  # x bounding-box diagonal, as in test_gpu_parity.py


def _create(s):
    L = _lib.load()
    X = _lib.f64(s.vertices)
    tets = _lib.i32(s.tets)
    rho, E, nu = _lib.f64(s.density), _lib.f64(s.youngs), _lib.f64(s.poisson)
    act = np.ascontiguousarray(s.active.astype(np.uint8))
    g = _lib.f64([0.0, 0.0, -9.81])
    h = ctypes.c_void_p()
    flags = _lib.MATERIAL_SNH | _lib.PRECISION_MIXED | _lib.MODE_GRAPH
    _lib.check(L.vbd_create(_lib.ptr(X, "d"), X.shape[0], _lib.ptr(tets, "i"), tets.shape[0],
                            _lib.ptr(rho, "d"), _lib.ptr(E, "d"), _lib.ptr(nu, "d"),
                            _lib.ptr(act, "u8"), 0.0, _lib.ptr(g, "d"), None, flags, 0, 0, 0,
                            ctypes.byref(h)), "vbd_create")
    return h


def _positions(h, n):
    out = np.empty((n, 3))
    _lib.check(_lib.load().vbd_get_positions(h, _lib.ptr(out, "d")))
    return out


def test_step_noalloc_matches_step_twice_in_a_row():
    L = _lib.load()
    s = scenes.cantilever(40)
    diag = float(np.linalg.norm(s.vertices.max(0) - s.vertices.min(0)))
    ref, na = _create(s), _create(s)
    try:
        for call in range(2):
            it_ref, it_na = ctypes.c_int(0), ctypes.c_int(0)
            _lib.check(L.vbd_step(ref, 1e-3, 1e-7, 1000, ctypes.byref(it_ref)), "vbd_step")
            _lib.check(L.vbd_step_noalloc(na, 1e-3, 1e-7, 1000, ctypes.byref(it_na)),
                       "vbd_step_noalloc")
            xr, xn = _positions(ref, s.n_vertices), _positions(na, s.n_vertices)
            assert np.isfinite(xn).all()
            assert np.abs(xn - xr).max() < POS_TOL * diag, (call, np.abs(xn - xr).max())
            assert it_na.value == it_ref.value, (call, it_na.value, it_ref.value)
            assert not np.array_equal(xn, s.vertices)   # the step moved the beam
            # the step's own kernel time and launch count: begin and end, and
            # per sweep one launch per colour plus the reduction and the check
            info = _lib.VBDInfo()
            _lib.check(L.vbd_get_info(na, ctypes.byref(info)))
            assert info.last_step_launches == 2 + it_na.value * (info.n_colors + 2), \
                (info.last_step_launches, it_na.value, info.n_colors)
            assert info.last_step_kernel_ms > 0.0
    finally:
        L.vbd_destroy(ref)
        L.vbd_destroy(na)
