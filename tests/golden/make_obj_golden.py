"""Generate the surface-mesh fixtures from the reference's own OBJ export.

Run by hand in a container that holds the reference checkout
(mmichelis/WarpVBD) at /root/reference.  It imports, unchanged,
src/_renderer.py (tet2obj :539-582, fix_tet_faces :466-485,
filter_unused_vertices :435-460; numpy only) and applies tet2obj to the
committed golden meshes (tests/golden/meshes.npz).

Output (committed): tests/golden/surfaces.npz with ``<name>/vertices`` and
``<name>/faces`` per mesh.

Run:  python tests/golden/make_obj_golden.py
"""
import os
import sys

import numpy as np

REF_SRC = "/root/reference/src"
HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["cantilever_20", "massspring_7_5", "ragged_6x5x4"]


def main():
    sys.path.insert(0, REF_SRC)
    import _renderer  # noqa: E402
    meshes = np.load(os.path.join(HERE, "meshes.npz"))
    out = {}
    for name in NAMES:
        v, f = _renderer.tet2obj(meshes[f"{name}/vertices"], meshes[f"{name}/tets"])
        out[f"{name}/vertices"] = np.asarray(v, np.float64)
        out[f"{name}/faces"] = np.asarray(f, np.int64)
        print(name, v.shape, f.shape)
    np.savez_compressed(os.path.join(HERE, "surfaces.npz"), **out)


if __name__ == "__main__":
    main()
