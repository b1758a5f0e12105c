"""Long-horizon FP64 oracle trajectories at the configured lengths.

Run by hand (CPU only; about two hours of 8 cores in all):

    python tests/golden/make_oracle_long.py [--cases c3 c160_snh c160_stvk c4]

The oracle (``oracle/vbd_oracle.c``, the FP64 C restatement of
mmichelis/WarpVBD ``src/vbd_solver.py``) is itself pinned to the reference's
own solver by ``ref_trajectories.npz``; the meshes come from
``warpvbd_b200.scenes``, whose mesher is pinned bit-exact to the reference's
``src/_utils.py`` by ``meshes.npz``.  These fixtures let the GPU tests compare
the CUDA solver with the oracle over whole trajectories that take the oracle
far too long to recompute in a test:

  c3         mass-spring, 11^3 cube under a 1x1x20 column (1 cm voxels), SNH
             E=5e5 nu=0.4 rho=1000, 1000 steps
  c160_snh   cantilever 160x16x16 (1.0 x 0.1 x 0.1 m), SNH E=1e6 nu=0.45
             rho=1000, 300 steps
  c160_stvk  the same beam, St. Venant-Kirchhoff, 100 steps
  c4         every 8th environment (32 of 256) of the 256-environment batch
             (warpvbd_b200.scenes.env_batch(256, seed=0)), 300 steps each

All: dt 1 ms, tol 1e-7, max 1000 sweeps, no damping, guarded Newton step (the
product's; it never triggers on these scenes).  Stored per case ``<name>/``:
``sweeps`` (per step), ``tip`` (tip-face mean displacement per step),
``sub`` (vertex ids kept), ``disp`` (float32 displacement x - X of those
vertices after the last step).  For c4 the arrays carry a leading
environment axis and ``envs`` lists the environment indices.
"""
import argparse
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _scene(name):
    from warpvbd_b200 import scenes
    if name == "c3":
        return scenes.mass_spring(11, 20), "snh", 1000, 1
    if name == "c160_snh":
        return scenes.cantilever(160), "snh", 300, 4
    if name == "c160_stvk":
        return scenes.cantilever(160), "stvk", 100, 4
    raise KeyError(name)


def run_single(s, material, steps, every, threads):
    from oracle import oracle
    oracle.set_threads(threads)
    o = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=1e-7,
                            max_iter=1000, material=material, guarded=True)
    sweeps, tip = [], []
    t0 = time.time()
    for k in range(steps):
        x = o.step(None, 1e-3)
        sweeps.append(o.last_iterations)
        tip.append((x[s.tip] - s.vertices[s.tip]).mean(0))
        if (k + 1) % 25 == 0:
            print(f"{s.name} {material}: step {k + 1}/{steps} ({time.time() - t0:.0f} s)",
                  flush=True)
    sub = np.arange(0, s.n_vertices, every, dtype=np.int32)
    return dict(sweeps=np.asarray(sweeps, np.int16), tip=np.asarray(tip),
                sub=sub, disp=(x[sub] - s.vertices[sub]).astype(np.float32))


def _c4_env(e):
    sys.path.insert(0, ROOT)
    from warpvbd_b200 import scenes
    s = scenes.env_batch(256, seed=0)[e]
    return e, run_single(s, "snh", 300, 8, 1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", nargs="*", default=["c3", "c160_snh", "c160_stvk", "c4"])
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--out", default=os.path.join(HERE, "oracle_long.npz"))
    args = ap.parse_args()
    sys.path.insert(0, ROOT)
    arrays = {}
    if os.path.exists(args.out):
        with np.load(args.out) as old:
            arrays.update({k: old[k] for k in old.files})
    for name in args.cases:
        if name == "c4":
            envs = list(range(0, 256, 8))
            with mp.get_context("spawn").Pool(args.threads) as pool:
                res = dict(pool.map(_c4_env, envs))
            arrays["c4/envs"] = np.asarray(envs, np.int32)
            for k in ("sweeps", "tip"):
                arrays[f"c4/{k}"] = np.stack([res[e][k] for e in envs])
            for k in ("sub", "disp"):  # ragged: concatenated with offsets
                arrays[f"c4/{k}"] = np.concatenate([res[e][k] for e in envs])
            arrays["c4/sub_offsets"] = np.cumsum([0] + [len(res[e]["sub"]) for e in envs])
        else:
            s, material, steps, every = _scene(name)
            out = run_single(s, material, steps, every, args.threads)
            for k, v in out.items():
                arrays[f"{name}/{k}"] = v
        np.savez_compressed(args.out, **arrays)
        print("wrote", name, flush=True)


if __name__ == "__main__":
    main()
