"""Accuracy and scaling sweeps of the solver (the counterpart of the
reference's benchmark scripts, benchmark_accuracy_vbd.py and the
tolerance study behind benchmark_accuracy_tolerance.png).

    python -m warpvbd_b200.sweeps --out sweeps.json [--quick]

Every row times the default solver (precision="fp64", the reference's
precision) and the fp32-arithmetic mode (precision="mixed") on the same mesh,
material, tolerance and steps, and gives the mixed run's error against the
FP64 one.

- resolution   cantilever 20x2x2 ... 320x32x32 (beam 1.0 x 0.1 x 0.1 m,
               x = 0 face fixed), Stable Neo-Hookean and St. Venant-Kirchhoff,
               E = 1 MPa, nu = 0.45, rho = 1000, dt = 1 ms, tol 1e-7.
               Reported per mesh: the largest vertex error over the run (per
               step, as a fraction of the bounding-box diagonal), the
               relative tip-face displacement error at the end, sweeps per
               step, simulated seconds per wall second and vertex updates per
               second.
- tolerance    the 160x16x16 SNH cantilever at tol 1e-5 ... 1e-9, against FP64
               at each tolerance and against FP64 at 1e-11 (the converged
               trajectory).
- mass_spring  the 11^3-voxel cube on a 1x1x20 column, 1000 steps, the
               bottom-face displacement against FP64.
- nsim         1 ... 4096 identical mass-spring systems in one batch: throughput
               (environment-seconds per wall second) and sweeps.
"""
import argparse
import json
import time

import numpy as np

from . import scenes


def _diag(X):
    return float(np.linalg.norm(X.max(0) - X.min(0)))


def _solver(s, **kw):
    from .vbd_solver import VBDSolver
    kw.setdefault("dx_tol", 1e-7)
    kw.setdefault("max_iter", 1000)
    kw.setdefault("tune", True)  # the autotuned launch shape (cached per mesh and precision)
    return VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, **kw)


def _pair_run(s, steps, dt=1e-3, tol=1e-7, material="snh", mode="auto", ref_tol=None,
              max_iter=1000, record=None):
    """Step the mixed-precision solver and its FP64 twin together; returns a
    dict of the mixed run's errors against the FP64 run, and sweeps and
    timing of both (wall time of each step with its positions download)."""
    import torch
    a = _solver(s, dx_tol=tol, material=material, mode=mode, max_iter=max_iter,
                precision="mixed")
    b = _solver(s, dx_tol=ref_tol or tol, material=material, mode=mode, precision="fp64",
                max_iter=max(max_iter, 20000 if ref_tol else max_iter))
    D = _diag(s.vertices)
    worst, its, its_b, t_mixed, t_fp64 = 0.0, [], [], 0.0, 0.0
    trace = []
    for k in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xa = a.step(a.old_positions, dt).numpy()
        t1 = time.perf_counter()
        xb = b.step(b.old_positions, dt).numpy()
        t_mixed += t1 - t0
        t_fp64 += time.perf_counter() - t1
        its.append(a.last_iterations)
        its_b.append(b.last_iterations)
        worst = max(worst, float(np.abs(xa - xb).max()) / D)
        if record is not None and k % record == 0:
            trace.append([k * dt, *((xa[s.tip] - s.vertices[s.tip]).mean(0).tolist()),
                          *((xb[s.tip] - s.vertices[s.tip]).mean(0).tolist())])
    da = (xa[s.tip] - s.vertices[s.tip]).mean(0)
    db = (xb[s.tip] - s.vertices[s.tip]).mean(0)
    k = np.bincount(s.tets.reshape(-1), minlength=s.n_vertices)
    solved = int((s.active & (k > 0)).sum())
    out = {"vertices": int(s.n_vertices), "tets": int(s.n_tets), "steps": steps,
           "mode": {0x100: "block", 0x200: "graph", 0x300: "hostloop", 0x400: "persist"}[
               a.info()["mode"]],
           "max_vertex_error_of_diag": worst,
           "tip_error_rel": float(np.linalg.norm(da - db) / max(np.linalg.norm(db), 1e-300)),
           "tip_displacement": da.tolist(), "tip_displacement_fp64": db.tolist(),
           "sweeps_mean": float(np.mean(its)), "sweeps_max": int(np.max(its)),
           "sim_s_per_wall_s": steps * dt / t_mixed,
           "vertex_updates_per_s": solved * float(np.sum(its)) / t_mixed,
           "fp64_mode": {0x100: "block", 0x200: "graph", 0x300: "hostloop", 0x400: "persist"}[
               b.info()["mode"]],
           "fp64_sweeps_mean": float(np.mean(its_b)),
           "fp64_sim_s_per_wall_s": steps * dt / t_fp64,
           "fp64_vertex_updates_per_s": solved * float(np.sum(its_b)) / t_fp64}
    if record is not None:
        out["trace"] = trace
    a.close()
    b.close()
    return out


def resolution(sizes=(20, 40, 80, 160, 320), materials=("snh", "stvk"), steps=300):
    res = {}
    for mat in materials:
        for n in sizes:
            s = scenes.cantilever(n)
            r = _pair_run(s, steps, material=mat)
            res[f"{mat}/{n}"] = r
            print(f"resolution {mat} {n}: {json.dumps({k: v for k, v in r.items() if k != 'trace'})}",
                  flush=True)
    return res


def tolerance(n=160, tols=(1e-5, 1e-6, 1e-7, 1e-8, 1e-9), steps=100):
    """Mixed precision and FP64 at each tolerance, both also compared with one
    FP64 run converged to tol 1e-11 (computed once)."""
    s = scenes.cantilever(n)
    D = _diag(s.vertices)
    truth = _solver(s, dx_tol=1e-11, precision="fp64", max_iter=20000)
    xt, t_sweeps = [], []
    for _ in range(steps):
        xt.append(truth.step(truth.old_positions, 1e-3).numpy())
        t_sweeps.append(truth.last_iterations)
    truth.close()
    res = {"converged_fp64_sweeps_mean": float(np.mean(t_sweeps))}
    dt_end = (xt[-1][s.tip] - s.vertices[s.tip]).mean(0)
    for tol in tols:
        r = _pair_run(s, steps, tol=tol)
        # replay the mixed run for the comparison with the converged trajectory
        a = _solver(s, dx_tol=tol, precision="mixed")
        worst = 0.0
        for k in range(steps):
            xa = a.step(a.old_positions, 1e-3).numpy()
            worst = max(worst, float(np.abs(xa - xt[k]).max()) / D)
        a.close()
        da = (xa[s.tip] - s.vertices[s.tip]).mean(0)
        r["tip_error_rel_vs_converged_fp64"] = float(np.linalg.norm(da - dt_end) /
                                                     np.linalg.norm(dt_end))
        r["max_vertex_error_of_diag_vs_converged_fp64"] = worst
        res[f"{tol:g}"] = r
        print(f"tolerance {tol:g}: {json.dumps(r)}", flush=True)
    return res


def mass_spring(steps=1000):
    s = scenes.mass_spring(11, 20)
    r = _pair_run(s, steps, record=10)
    print(f"mass_spring: {json.dumps({k: v for k, v in r.items() if k != 'trace'})}",
          flush=True)
    return r


def nsim(counts=(1, 4, 16, 64, 256, 1024, 4096), steps=20, warmup=3):
    import torch
    from .batched import BatchedVBDSolver
    base = scenes.mass_spring(11, 20)
    res = {}
    for n in counts:
        sol = BatchedVBDSolver([base] * n, dx_tol=1e-7, max_iter=1000, tpv=2,
                               block_threads=512, cluster=4, tiered=n > 1)
        for _ in range(warmup):
            sol.step(1e-3)
        st = torch.cuda.ExternalStream(sol.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = []
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(steps):
            sol.step(1e-3, blocking=False)
            its.append(np.max(sol.sync()))
        b.record(st)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / steps
        res[str(n)] = {"ms_per_step": ms, "env_sim_s_per_wall_s": n * 1e-3 / (ms * 1e-3),
                       "sweeps_mean": float(np.mean(its)),
                       "vertices": int(n * base.n_vertices)}
        print(f"nsim {n}: {json.dumps(res[str(n)])}", flush=True)
        sol.close()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default="sweeps.json")
    ap.add_argument("--quick", action="store_true", help="fewer steps and sizes (smoke run)")
    ap.add_argument("--only", default="resolution,tolerance,mass_spring,nsim")
    a = ap.parse_args(argv)
    parts = a.only.split(",")
    out = {}
    if "resolution" in parts:
        out["resolution"] = resolution(sizes=(20, 40) if a.quick else (20, 40, 80, 160, 320),
                                       steps=20 if a.quick else 300)
    if "tolerance" in parts:
        out["tolerance"] = tolerance(n=40 if a.quick else 160, steps=10 if a.quick else 100)
    if "mass_spring" in parts:
        out["mass_spring"] = mass_spring(steps=50 if a.quick else 1000)
    if "nsim" in parts:
        out["nsim"] = nsim(counts=(1, 4, 16) if a.quick else (1, 4, 16, 64, 256, 1024, 4096))
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    return out


if __name__ == "__main__":
    main()
