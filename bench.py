"""Benchmark of the VBD time step on B200.

Default workload: the 160x16x16 Stable Neo-Hookean cantilever (1.0 x 0.1 x
0.1 m beam, 46,529 vertices, 204,800 tets; E=1e6 Pa, nu=0.45, rho=1000, x=0
face fixed, gravity -z, dt=1 ms, tol 1e-7, max 1000 sweeps), plain VBD in
fp32.  A "step" is one implicit-Euler time step (inertia guess, colour sweeps
until max|dx_x+dx_y+dx_z| < tol, velocity update).  value = simulated
seconds per wall second, summed over ranks (each rank runs its own replica:
weak scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # the FP64 CPU oracle on the host cores

Timing: every timed step is bracketed by CUDA events on the solver's stream,
with a 256 MiB write between steps to flush L2; the e2e figure runs the same
steps through the public Python API with host arrays (positions uploaded
before and downloaded after every step).
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from warpvbd_b200 import scenes  # noqa: E402

DT = 1e-3
TOL = 1e-7
MAX_ITER = 1000


def workload(name):
    if name == "cantilever160":
        return scenes.cantilever(160), "cantilever 160x16x16 SNH fp32"
    if name == "cantilever80":
        return scenes.cantilever(80), "cantilever 80x8x8 SNH fp32"
    if name == "cantilever320":
        return scenes.cantilever(320), "cantilever 320x32x32 SNH fp32"
    if name == "cantilever20":
        return scenes.cantilever(20), "cantilever 20x2x2 SNH fp32"
    if name == "massspring":
        return scenes.mass_spring(11, 20), "mass-spring 11^3 cube + 1x1x20 column SNH fp32"
    raise SystemExit(f"unknown workload {name}")


def bytes_per_sweep(s):
    """Algorithmic bytes of one sweep: sum over solved vertices of 44 + 104 k_v
    (fp32 state 44 B per vertex, 104 B per incident tet)."""
    k = np.bincount(s.tets.reshape(-1), minlength=s.n_vertices)
    solved = s.active & (k > 0)
    return float((44 + 104 * k[solved]).sum()), int(solved.sum())


def clocks_start():
    try:
        f = open(os.path.join(ROOT, "gpurun_out", "clocks_bench.csv") if os.path.isdir(
            os.path.join(ROOT, "gpurun_out")) else os.devnull, "w")
        p = subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        return p, f
    except Exception:
        return None, None


def clocks_stop(p, f, gpu_index):
    if p is None:
        return None
    p.terminate()
    try:
        out, _ = p.communicate(timeout=5)
    except Exception:
        p.kill()
        out = ""
    if f:
        f.write(out)
        f.close()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        c = [x.strip() for x in line.split(",")]
        if len(c) < 9 or c[0] != str(gpu_index):
            continue
        try:
            sm.append(float(c[1]))
            mx.append(float(c[2]))
        except ValueError:
            continue
        for n, v in zip(names, c[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
            "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(s, steps_budget_s=20.0, max_steps=50):
    """Time the FP64 oracle (OpenMP, all host threads) on whole steps of the
    same workload; returns sim-s/wall-s and the sample description."""
    from oracle import oracle
    n = oracle.max_threads()
    oracle.set_threads(n)
    o = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=TOL,
                            max_iter=MAX_ITER, guarded=True)
    t0 = time.perf_counter()
    k = 0
    while k < max_steps and (time.perf_counter() - t0) < steps_budget_s:
        o.step(None, DT)
        k += 1
    el = time.perf_counter() - t0
    return {"value": k * DT / el, "unit": "sim-s/wall-s", "cores": n, "kind": "port",
            "sample": f"first {k} steps of the same workload, FP64 C oracle, OpenMP {n} threads"}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def run_reference(args, s, desc):
    world, rank, _ = dist_init()
    if rank != 0:
        return
    from oracle import oracle
    n = oracle.max_threads()
    oracle.set_threads(n)
    o = oracle.OracleSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=TOL,
                            max_iter=MAX_ITER, guarded=True)
    budget = args.reference_budget_s
    for _ in range(args.warmup):
        o.step(None, DT)
    t0 = time.perf_counter()
    k = 0
    while k < args.steps and (time.perf_counter() - t0) < budget:
        o.step(None, DT)
        k += 1
    el = time.perf_counter() - t0
    v = k * DT / el
    line = {"impl": "reference", "metric": "sim-s/wall-s", "value": v, "unit": "sim-s/wall-s",
            "n_gpus": args.gpus, "steps": k, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "dt": DT, "tol": TOL, "max_iter": MAX_ITER,
                       "vertices": s.n_vertices, "tets": s.n_tets},
            "cpu_baseline": {"value": v, "unit": "sim-s/wall-s", "cores": n, "kind": "port",
                             "sample": f"{k} whole steps after {args.warmup} warm-up steps "
                                       "(FP64 C restatement of the reference; Warp is not "
                                       "installable offline)"},
            "e2e": {"value": v, "unit": "sim-s/wall-s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, s, desc):
    import torch
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    from warpvbd_b200 import VBDSolver
    sol = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=TOL, max_iter=MAX_ITER,
                    device=f"cuda:{local}", mode=args.mode)
    info = sol.info()
    stream = torch.cuda.ExternalStream(sol.stream, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    # warm-up (graph instantiation happens here)
    for _ in range(args.warmup):
        sol.step(sol.old_positions, DT)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    iters = []
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk, clkf = clocks_start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xFF)
            evs[k][0].record(stream)
        sol.step(sol.old_positions, DT, blocking=False)
        evs[k][1].record(stream)
        iters.append(None)
        sol.sync()
        iters[-1] = sol.last_iterations
    torch.cuda.synchronize()
    clocks = clocks_stop(clk, clkf, local)
    step_ms = np.array([a.elapsed_time(b) for a, b in evs])
    total_ms = float(step_ms.sum())
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    iters = np.array(iters)
    value = world * args.steps * DT / (total_ms * 1e-3)

    # end to end through the public API with host arrays
    x_host = sol.old_positions.numpy()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        x_host = sol.step(x_host, DT).numpy()
    e2e_s = time.perf_counter() - t0
    e2e = world * args.e2e_steps * DT / e2e_s

    bsweep, nsolved = bytes_per_sweep(s)
    peak, peak_kind = measured_peak()
    mode = {0x100: "block", 0x200: "graph", 0x300: "hostloop"}[info["mode"]]
    achieved = bsweep * iters.sum() / (total_ms * 1e-3) / 1e9
    if mode == "block":
        launches = args.steps
    else:
        launches = int(args.steps * 2 + iters.sum() * (info["n_colors"] + 1))
    line = {"metric": "sim-s/wall-s", "value": value, "unit": "sim-s/wall-s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "dt": DT, "tol": TOL, "max_iter": MAX_ITER,
                       "vertices": s.n_vertices, "tets": s.n_tets, "mode": mode,
                       "tpv": info["tpv"], "block_threads": info["block_threads"],
                       "parallelism": f"replicas x{world}",
                       "l2": "256 MiB buffer written between timed steps"},
            "iters_per_step": {"mean": float(iters.mean()), "min": int(iters.min()),
                               "max": int(iters.max())},
            "vertex_updates_per_s": world * nsolved * float(iters.sum()) / (total_ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_sweep": bsweep},
            "e2e": {"value": e2e, "unit": "sim-s/wall-s",
                    "h2d_bytes_per_step": 24 * s.n_vertices,
                    "d2h_bytes_per_step": 24 * s.n_vertices},
            "gpu_launches": launches}
    if clocks:
        line["clocks"] = clocks
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(s, args.cpu_budget_s)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cantilever160")
    ap.add_argument("--mode", default="auto", choices=["auto", "block", "graph", "hostloop"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--reference-budget-s", type=float, default=150.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    s, desc = workload(args.workload)
    if args.impl == "reference":
        run_reference(args, s, desc)
    else:
        run_ours(args, s, desc)


if __name__ == "__main__":
    main()
