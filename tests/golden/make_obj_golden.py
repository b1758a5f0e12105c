"""Generate the surface-mesh fixtures from the reference's own OBJ export.

Run by hand in a container that holds a checkout of the reference
(mmichelis/WarpVBD).  It imports, unchanged,
src/_renderer.py (tet2obj :539-582, fix_tet_faces :466-485,
filter_unused_vertices :435-460; numpy only) and applies tet2obj to the
committed golden meshes (tests/golden/meshes.npz).

Output (committed): tests/golden/surfaces.npz with ``<name>/vertices`` and
``<name>/faces`` per mesh.

Run:  python tests/golden/make_obj_golden.py --ref <checkout>
      (``--ref`` defaults to the environment variable WARPVBD_REFERENCE)
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["cantilever_20", "massspring_7_5", "ragged_6x5x4"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("WARPVBD_REFERENCE"),
                    help="checkout of mmichelis/WarpVBD (default: $WARPVBD_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set WARPVBD_REFERENCE")
    sys.path.insert(0, os.path.join(os.path.abspath(args.ref), "src"))
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
