"""Generate the golden mesh / colouring fixtures from the reference's own code.

This script is run by hand in a container that holds a checkout of the
reference (mmichelis/WarpVBD).  It imports, unchanged:

  * src/_utils.py     voxel2hex (:35-89), hex2tets (:92-108)
  * src/coloring.py   compute_adjacency_dict (:24-38), graph_coloring (:40-72)

``coloring.py:3`` does ``import warp`` but the two functions used never touch
it, so a stub module is registered under ``sys.modules['warp']`` first.

Outputs (committed):
  tests/golden/meshes.npz   full vertex / tet / colour arrays for the small
                            meshes (prefix ``<name>/``)
  tests/golden/hashes.json  sha256 of the same arrays plus colour-group sizes
                            for every mesh, including the large cantilevers
                            whose arrays are too big to commit.

Run:  python tests/golden/make_golden.py --ref <checkout> [--large]
      (``--ref`` defaults to the environment variable WARPVBD_REFERENCE)
"""
import argparse
import hashlib
import io
import json
import os
import sys
import types
import contextlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference(ref_src):
    sys.modules.setdefault("warp", types.ModuleType("warp"))
    sys.path.insert(0, ref_src)
    import _utils as ref_utils  # noqa: E402
    import coloring as ref_coloring  # noqa: E402
    return ref_utils, ref_coloring


def mesh_specs(large):
    """Name -> (voxel bool array, (dx, dy, dz)).  Same geometry builders as
    warpvbd_b200.scenes, written out independently here."""
    specs = {}
    for n in [20, 40] + ([80, 160, 320] if large else [80]):
        vox = np.ones((n, n // 10, n // 10), dtype=bool)
        h = 1.0 / n
        specs[f"cantilever_{n}"] = (vox, (h, h, h))
    # mass-spring: cube of `cube` voxels hanging from a 1x1x`col` column
    for cube, col in [(11, 20), (7, 5), (15, 30), (9, 13)]:
        vox = np.zeros((cube, cube, cube + col), dtype=bool)
        vox[:, :, :cube] = True
        vox[cube // 2, cube // 2, cube:] = True
        specs[f"massspring_{cube}_{col}"] = (vox, (0.01, 0.01, 0.01))
    # a ragged voxel set (holes, overhangs) to exercise the mesher's flags
    rng = np.random.default_rng(1234)
    vox = rng.random((6, 5, 4)) < 0.6
    specs["ragged_6x5x4"] = (vox, (0.02, 0.03, 0.05))
    return specs


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--large", action="store_true",
                    help="also hash the 160x16x16 and 320x32x32 cantilevers")
    ap.add_argument("--ref", default=os.environ.get("WARPVBD_REFERENCE"),
                    help="checkout of mmichelis/WarpVBD (default: $WARPVBD_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set WARPVBD_REFERENCE")
    ref_utils, ref_coloring = _import_reference(os.path.join(os.path.abspath(args.ref), "src"))

    arrays = {}
    hashes = {}
    for name, (vox, d) in mesh_specs(args.large).items():
        verts, hexes = ref_utils.voxel2hex(vox, *d)
        tets = ref_utils.hex2tets(hexes)
        with contextlib.redirect_stdout(io.StringIO()):
            adjacency, max_deg = ref_coloring.compute_adjacency_dict(tets)
            coloring, groups = ref_coloring.graph_coloring(adjacency)
        verts = np.asarray(verts, dtype=np.float64)
        tets32 = np.asarray(tets, dtype=np.int32)
        col32 = np.asarray(coloring, dtype=np.int32)
        sizes = [len(groups[c]) for c in range(len(groups))]
        hashes[name] = {
            "voxels_shape": list(vox.shape),
            "voxels_sha256": sha(vox.astype(np.uint8)),
            "spacing": list(d),
            "n_vertices": int(verts.shape[0]),
            "n_tets": int(tets32.shape[0]),
            "max_degree": int(max_deg),
            "color_group_sizes": sizes,
            "vertices_sha256": sha(verts),
            "tets_sha256": sha(tets32),
            "coloring_sha256": sha(col32),
        }
        if verts.shape[0] <= 7000:
            arrays[f"{name}/vertices"] = verts
            arrays[f"{name}/tets"] = tets32
            arrays[f"{name}/coloring"] = col32
            if name.startswith("ragged"):
                arrays[f"{name}/voxels"] = vox
        print(name, verts.shape[0], tets32.shape[0], sizes)

    np.savez_compressed(os.path.join(HERE, "meshes.npz"), **arrays)
    old = {}
    path = os.path.join(HERE, "hashes.json")
    if os.path.exists(path) and not args.large:
        with open(path) as f:
            old = json.load(f)
    old.update(hashes)
    with open(path, "w") as f:
        json.dump(old, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
