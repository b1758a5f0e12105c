"""Golden time-step trajectories from the reference's own solver code.

Run by hand in a container that holds a checkout of mmichelis/WarpVBD:

    python tests/golden/make_ref_trajectories.py --ref <checkout> [--jobs 6]

(``--ref`` defaults to the environment variable WARPVBD_REFERENCE).  It imports
the checkout's ``src/vbd_solver.py`` UNCHANGED, with the pure-Python Warp
stand-in ``warp_standin.py`` registered as ``sys.modules['warp']`` (warp-lang
1.10.0 cannot be installed offline) and a stub ``matplotlib`` (imported at
``vbd_solver.py:4``, used only by a disabled plot).  Meshes come from the
checkout's own ``src/_utils.py`` (voxel2hex, hex2tets), the colouring from
its ``src/coloring.py`` (called by ``VBDSolver.__init__``).  Every case drives
the solver exactly as ``examples/run_cantilever.py:83-84`` does:
``solution = solver.step(solver.old_positions, wp.float64(dt))``.

The StVK case runs an edited copy of the file in a temporary directory: the
Stable Neo-Hookean block (``vbd_solver.py:107-124``) commented out and the
commented St. Venant-Kirchhoff block (``:127-144``) restored, nothing else
changed.

Sweep counts: the step's iteration index is local to ``step``, so it is read
off the number of ``accumulate_grad_hess`` launches (one per colour and
sweep, ``vbd_solver.py:552-565``).  The non-convergence warning
(``:581-582``) is captured from stdout.

Output (committed): ``tests/golden/ref_trajectories.npz`` with, per case
``<name>/``: ``sweeps`` [steps], ``warned`` [steps], ``final_dx`` [steps] (the
value the warning prints, NaN without a warning), ``rec_steps`` (1-based
step numbers recorded), ``positions`` [len(rec_steps), V, 3] (float64),
``params`` (a JSON string: mesh, material, dt, tol, max_iter, damping), plus
``vertices`` / ``tets`` / ``active`` / ``color_groups`` / ``adj_v2e`` as the
reference built them.  Cases run in parallel processes (one per case).
"""
import argparse
import contextlib
import io
import json
import multiprocessing as mp
import os
import re
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# name -> case description.  "record": every step up to `dense`, then every
# `every`-th step and the last one.
CASES = {
    # cantilever 20x2x2 (1.0 x 0.1 x 0.1 m, 5 cm voxels), SNH E=1e6 nu=0.45
    # rho=1000, x=0 face fixed, no damping, dt 1 ms, tol 1e-7, max 1000 sweeps
    "cantilever20_snh": dict(scene="cantilever", nx=20, material="snh", kd=0.0, steps=300,
                             dense=30, every=10),
    "cantilever20_stvk": dict(scene="cantilever", nx=20, material="stvk", kd=0.0, steps=100,
                              dense=30, every=10),
    # the reference's default damping coefficient (vbd_solver.py:375)
    "cantilever20_damped": dict(scene="cantilever", nx=20, material="snh", kd=1.0, steps=40,
                                dense=40, every=10),
    # max_iter exhausted every step: the warning path and a truncated solve
    "cantilever20_maxiter3": dict(scene="cantilever", nx=20, material="snh", kd=0.0, steps=8,
                                  dense=8, every=1, max_iter=3),
    # a mass-spring: 5^3 cube of 1 cm voxels under a 1x1x6 column, top fixed,
    # E=5e5 nu=0.4 rho=1000
    "massspring5_6": dict(scene="massspring", cube=5, col=6, material="snh", kd=0.0, steps=60,
                          dense=30, every=10),
}


def _stub_modules(ref_src):
    import warp_standin
    sys.modules["warp"] = warp_standin
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.path.insert(0, ref_src)


def _stvk_copy(ref_src, dst_dir):
    """vbd_solver.py with the SNH block (107-124) commented and the StVK block
    (127-144) restored; nothing else touched."""
    with open(os.path.join(ref_src, "vbd_solver.py")) as f:
        lines = f.read().split("\n")
    snh = range(106, 124)   # 0-based rows of lines 107-124
    stvk = range(126, 144)  # lines 127-144
    assert lines[106].strip().startswith("### Stable Neo-Hookean"), lines[106]
    assert lines[126].strip().startswith("### St. Venant-Kirchhoff"), lines[126]
    for r in snh:
        if lines[r].strip():
            lines[r] = "#" + lines[r]
    for r in stvk:
        lines[r] = re.sub(r"^(\s*)# ?", r"\1", lines[r], count=1) if lines[r].strip() else lines[r]
    path = os.path.join(dst_dir, "vbd_solver_stvk.py")
    with open(path, "w") as f:
        f.write("\n".join(lines))
    return path


def _scene(ref_utils, c):
    if c["scene"] == "cantilever":
        nx = c["nx"]
        h = 1.0 / nx
        vox = np.ones((nx, nx // 10, nx // 10), dtype=bool)
        X, hexes = ref_utils.voxel2hex(vox, h, h, h)
        tets = ref_utils.hex2tets(hexes)
        active = ~(X[:, 0] < 1e-3)   # examples/run_cantilever.py:41-44
        E, nu, rho = 1e6, 0.45, 1000.0
    else:
        cube, col = c["cube"], c["col"]
        vox = np.zeros((cube, cube, cube + col), dtype=bool)
        vox[:, :, :cube] = True
        vox[cube // 2, cube // 2, cube:] = True
        X, hexes = ref_utils.voxel2hex(vox, 0.01, 0.01, 0.01)
        tets = ref_utils.hex2tets(hexes)
        top = (cube + col) * 0.01
        active = ~(X[:, 2] > top - 1e-4)
        E, nu, rho = 5e5, 0.4, 1000.0
    return np.asarray(X, np.float64), np.asarray(tets, np.int32), active, E, nu, rho


def run_case(args):
    name, ref_src = args
    c = dict(CASES[name])
    sys.path.insert(0, HERE)
    _stub_modules(ref_src)
    import warp_standin as wp
    import _utils as ref_utils
    if c["material"] == "stvk":
        tmp = tempfile.mkdtemp()
        _stvk_copy(ref_src, tmp)
        sys.path.insert(0, tmp)
        import vbd_solver_stvk as ref
    else:
        import vbd_solver as ref
    X, tets, active, E, nu, rho = _scene(ref_utils, c)
    T = tets.shape[0]
    dt, tol, max_iter = 1e-3, 1e-7, c.get("max_iter", 1000)
    with contextlib.redirect_stdout(io.StringIO()):
        solver = ref.VBDSolver(
            initial_positions=wp.array(X, dtype=wp.vec3d, device="cpu"),
            elements=wp.array(tets, dtype=wp.vec4i, device="cpu"),
            densities=wp.array(rho * np.ones(T), dtype=wp.float64, device="cpu"),
            youngs_modulus=wp.array(E * np.ones(T), dtype=wp.float64, device="cpu"),
            poissons_ratio=wp.array(nu * np.ones(T), dtype=wp.float64, device="cpu"),
            damping_coefficient=c["kd"],
            active_mask=wp.array(active, dtype=wp.bool, device="cpu"),
            gravity=wp.vec3d(0.0, 0.0, -9.81),
            dx_tol=tol, max_iter=max_iter, device="cpu")
    n_colors = solver.color_groups.shape[0]
    steps = c["steps"]
    rec = [k for k in range(1, steps + 1)
           if k <= c["dense"] or k % c["every"] == 0 or k == steps]
    sweeps, warned, final_dx, pos = [], [], [], []
    t0 = time.time()
    for k in range(1, steps + 1):
        n0 = wp.launch_counts.get("accumulate_grad_hess", 0)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            sol = solver.step(solver.old_positions, wp.float64(dt))
        n1 = wp.launch_counts.get("accumulate_grad_hess", 0)
        assert (n1 - n0) % n_colors == 0
        sweeps.append((n1 - n0) // n_colors)
        text = buf.getvalue()
        warned.append("did not converge" in text)
        m = re.search(r"Final dx max: (\S+)", text)
        final_dx.append(float(m.group(1)) if m else float("nan"))
        if k in rec:
            pos.append(sol.numpy().copy())
        if k % 10 == 0:
            print(f"{name}: step {k}/{steps} sweeps {sweeps[-1]} "
                  f"({time.time() - t0:.0f} s)", flush=True)
    params = dict(c)
    params.update(case=name, dt=dt, tol=tol, max_iter=max_iter, E=E, nu=nu, rho=rho,
                  n_colors=int(n_colors))
    out = {
        "sweeps": np.asarray(sweeps, np.int32),
        "warned": np.asarray(warned, bool),
        "final_dx": np.asarray(final_dx, np.float64),
        "rec_steps": np.asarray(rec, np.int32),
        "positions": np.asarray(pos, np.float64),
        "params": np.asarray(json.dumps(params, sort_keys=True)),
        "vertices": X,
        "tets": tets,
        "active": active,
        "color_groups": solver.color_groups.numpy().astype(np.int32),
        "adj_v2e": solver.adj_v2e.numpy().astype(np.int32),
    }
    return name, out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("WARPVBD_REFERENCE"),
                    help="checkout of mmichelis/WarpVBD (default: $WARPVBD_REFERENCE)")
    ap.add_argument("--jobs", type=int, default=len(CASES))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--out", default=os.path.join(HERE, "ref_trajectories.npz"))
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set WARPVBD_REFERENCE")
    ref_src = os.path.join(os.path.abspath(args.ref), "src")
    ctx = mp.get_context("spawn")
    arrays = {}
    if os.path.exists(args.out):
        with np.load(args.out) as old:
            arrays.update({k: old[k] for k in old.files})
    with ctx.Pool(min(args.jobs, len(args.cases))) as pool:
        # each case is written as soon as it is done
        for name, out in pool.imap_unordered(run_case, [(n, ref_src) for n in args.cases]):
            for k, v in out.items():
                arrays[f"{name}/{k}"] = v
            np.savez_compressed(args.out, **arrays)
            print("wrote", name, flush=True)


if __name__ == "__main__":
    main()
