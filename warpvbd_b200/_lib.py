"""ctypes binding of libvbd_b200.so (the C ABI in include/vbd_b200.h).

The library is built in-tree (``make -C warpvbd_b200/csrc``, or
``warpvbd_b200.build()``).  There is no CPU fallback: importing a solver
without the compiled library raises ``ImportError``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# WARPVBD_B200_LIB selects another build of the library, e.g. the
# bounds-checked libvbd_b200_check.so (`make -C warpvbd_b200/csrc check`)
LIB_PATH = os.environ.get("WARPVBD_B200_LIB") or os.path.join(_HERE, "libvbd_b200.so")
CSRC = os.path.join(_HERE, "csrc")

# status codes
OK = 0
NOT_CONVERGED = 1
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_SINGULAR_DM = -3
ERR_TOO_MANY_COLORS = -4
ERR_NONFINITE = -5
ERR_TIMEOUT = -6
ERR_NO_DEVICE = -7
ERR_UNSUPPORTED = -8
ERR_BOUNDS = -9

# flags
MATERIAL_SNH = 0x0
MATERIAL_STVK = 0x1
PRECISION_FP32 = 0x00
PRECISION_FP64 = 0x10
PRECISION_MIXED = 0x20
PRECISIONS = {"fp32": PRECISION_FP32, "mixed": PRECISION_MIXED, "fp64": PRECISION_FP64}
GPU_SETUP = 0x40
MODE_AUTO = 0x000
MODE_BLOCK = 0x100
MODE_GRAPH = 0x200
MODE_HOSTLOOP = 0x300
ORDER_INDEX = 0x1000
STRICT_SPD = 0x2000
TIERED = 0x4000
TIERED_WIDE = 0x80
PERSIST_GRID_BARRIERS = 0x8000
CLUSTER_SHIFT = 16
MAX_CLUSTER = 16


def cluster_flags(cluster):
    """The flag bits of a block-mode cluster size: 0 (automatic) or 1 to 16
    thread blocks per cluster; anything else raises ValueError (the field
    is 5 bits wide, so a larger value must not be shifted in)."""
    c = int(cluster)
    if c != cluster or not 0 <= c <= MAX_CLUSTER:
        raise ValueError(f"cluster must be an integer from 0 (automatic) to {MAX_CLUSTER}, "
                         f"got {cluster!r}")
    return c << CLUSTER_SHIFT

MODE_PERSIST = 0x400
MODES = {"auto": MODE_AUTO, "block": MODE_BLOCK, "graph": MODE_GRAPH, "hostloop": MODE_HOSTLOOP,
         "persist": MODE_PERSIST}

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class VBDInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "n_vertices", "n_tets", "n_env", "n_colors", "max_valence", "mode", "tpv",
        "block_threads", "precision", "material")] + [
        ("n_slots", ctypes.c_longlong), ("n_slot_records", ctypes.c_longlong),
        ("device_bytes", ctypes.c_longlong), ("n_unique_records", ctypes.c_int),
        ("record_format", ctypes.c_int), ("cluster", ctypes.c_int), ("n_blocks", ctypes.c_int),
        ("last_step_launches", ctypes.c_int), ("last_step_kernel_ms", ctypes.c_float)]


# every entry point declared in include/vbd_b200.h: name -> (restype, argtypes)
SIGNATURES = {
    "vbd_version": (ctypes.c_int, []),
    "vbd_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "vbd_last_error_message": (ctypes.c_char_p, []),
    "vbd_device_count": (ctypes.c_int, []),
    "vbd_graph_coloring": (ctypes.c_int, [_i, ctypes.c_int, _i, _ip, _ip]),
    "vbd_graph_coloring_gpu": (ctypes.c_int, [_i, ctypes.c_int, _i, _ip, _ip, ctypes.c_int]),
    "vbd_create": (ctypes.c_int, [_d, ctypes.c_int, _i, ctypes.c_int, _d, _d, _d, _u8,
                                  ctypes.c_double, _d, _i, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "vbd_create_batched": (ctypes.c_int, [_d, ctypes.c_int, _i, ctypes.c_int, _d, _d, _d, _u8,
                                          ctypes.c_double, _d, _i, _i, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.POINTER(_vp)]),
    "vbd_destroy": (None, [_vp]),
    "vbd_reset": (ctypes.c_int, [_vp]),
    "vbd_set_wait_limits": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_ulonglong]),
    "vbd_set_trace": (ctypes.c_int, [_vp, ctypes.c_int]),
    "vbd_get_trace": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int,
                                     _ip]),
    "vbd_ws_vertex_rows": (ctypes.c_int, [_vp, _i]),
    "vbd_incremental_potential": (ctypes.c_int, [_vp, ctypes.c_double, _d, _d]),
    "vbd_step": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _ip]),
    "vbd_step_batched": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _d,
                                        ctypes.c_int, _ip]),
    "vbd_step_batched_to": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _d,
                                           ctypes.c_int, _ip, _d]),
    "vbd_sync": (ctypes.c_int, [_vp]),
    "vbd_get_iterations": (ctypes.c_int, [_vp, _ip]),
    "vbd_get_final_dx": (ctypes.c_int, [_vp, _d]),
    "vbd_get_positions": (ctypes.c_int, [_vp, _d]),
    "vbd_set_positions": (ctypes.c_int, [_vp, _d]),
    "vbd_get_velocities": (ctypes.c_int, [_vp, _d]),
    "vbd_set_velocities": (ctypes.c_int, [_vp, _d]),
    "vbd_get_color_groups": (ctypes.c_int, [_vp, _i, _ip, _ip]),
    "vbd_get_info": (ctypes.c_int, [_vp, ctypes.POINTER(VBDInfo)]),
    "vbd_get_stream": (_vp, [_vp]),
    "vbd_step_noalloc": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        _ip]),
    "vbd_ws_param_count": (ctypes.c_int, []),
    "vbd_ws_feature_width": (ctypes.c_int, []),
    "vbd_set_warmstart": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_float)]),
    "vbd_ws_features": (ctypes.c_int, [_vp, ctypes.c_double, _vp]),
    "vbd_ws_targets": (ctypes.c_int, [_vp, _vp, _vp]),
    "vbd_ws_predict": (ctypes.c_int, [_vp, _vp, _vp]),
    "vbd_get_env_status": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint32)]),
    "vbd_mlp_train_batch": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                           _vp]),
    "vbd_mlp_forward": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "vbd_mlp_train_scratch_floats": (ctypes.c_size_t, [ctypes.c_int]),
    "vbd_mlp_adam": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                    _vp]),
}

_lib = None


def build(verbose=False):
    """Compile libvbd_b200.so for sm_100a in place (nvcc, no GPU needed)."""
    cmd = ["make", "-C", CSRC] + ([] if verbose else ["-s"])
    subprocess.check_call(cmd)


def load():
    """Load the compiled library (raises ImportError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C {CSRC}` (nvcc, sm_100a). "
            "warpvbd_b200 has no CPU fallback.")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class VBDError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        super().__init__(f"{message} (status {status})" if message else f"status {status}")


def check(status, what=""):
    """Raise on negative status codes; return the code otherwise."""
    if status < 0:
        L = load()
        msg = L.vbd_last_error_message().decode(errors="replace")
        text = L.vbd_status_string(status).decode()
        raise VBDError(status, f"{what}: {text}: {msg}".strip(": "))
    return status


def ptr(a, kind):
    if a is None:
        return None
    return a.ctypes.data_as({"d": _d, "i": _i, "u8": _u8}[kind])


def f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(shape) if shape is not None else a


def i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))
