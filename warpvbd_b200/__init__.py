"""warpvbd_b200: Vertex Block Descent for tetrahedral soft bodies on B200 (sm_100a).

A drop-in for the time-step solve of mmichelis/WarpVBD (src/vbd_solver.py):
``VBDSolver`` keeps the reference's constructor / ``step`` / ``reset``
interface and runs hand-written CUDA kernels from ``libvbd_b200.so`` through
a C ABI (include/vbd_b200.h).  ``BatchedVBDSolver`` steps many uneven
environments in one launch with per-environment convergence.
"""
from . import mesh, scenes
from ._lib import build, load, VBDError
from .mesh import voxel2hex, hex2tets

__all__ = ["mesh", "scenes", "build", "load", "VBDError", "voxel2hex", "hex2tets",
           "VBDSolver", "BatchedVBDSolver"]


def __getattr__(name):
    # the solver classes need the compiled library; import them lazily so the
    # mesher and scenes stay usable on machines without the .so
    if name == "VBDSolver":
        from .vbd_solver import VBDSolver
        return VBDSolver
    if name == "BatchedVBDSolver":
        from .batched import BatchedVBDSolver
        return BatchedVBDSolver
    raise AttributeError(name)
