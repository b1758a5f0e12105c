"""Benchmark of the VBD time step on B200.

Default workload (``--workload batch256``): 256 mass-spring environments of
uneven size drawn from seed 0 (cube edge 7-15 voxels, column 5-30 voxels,
1 cm voxels, E log-uniform 1e5-1e6 Pa, nu 0.35-0.48, rho 1000, the column's
top face fixed, gravity -z), Stable Neo-Hookean, dt = 1 ms, tol 1e-7, at most
1000 sweeps per step, 1000 steps; arithmetic and state in fp64 (the
reference's precision; ``--precision mixed`` for fp32 per-slot arithmetic).
All environments advance in one launch per step, each with its own
convergence test.

A "step" is one implicit-Euler time step of every environment (inertia guess,
colour sweeps until max|dx_x+dx_y+dx_z| < tol, velocity update).
value = simulated environment-seconds per wall second, summed over ranks
(each rank steps its own copy of the batch: weak scaling, no collective on
the data path).  Other workloads: cantilever20/40/80/160/320, massspring.
The headline batched run starts every step from the learned warm start (the
metric's "warm-start + batched" form); plain batched VBD is timed beside it
(``plain_batched``, with the ratio; ``--warmstart off`` swaps the two).

The cost of a step changes along the 1000-step trajectory (the sweep counts
grow over the first few hundred steps as the environments swing), so the
timed window does not start from rest: every timed run first advances its
solver ``--start-step`` steps (default 500, the middle of the trajectory)
untimed, then takes the warm-up and timed steps.  ``batch_1000_steps``
reports the whole trajectory from rest, plain and warm-started, every step
device-timed, with each environment's tip displacement every 100 steps: the
warm-started run's against plain VBD's at the same tolerance, and both
against a plain run at tol 1e-9 (the accuracy each form buys at tol 1e-7).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # FP64 CPU oracle on the host cores

Timing: each timed step is bracketed by CUDA events on the solver's stream;
a 256 MiB buffer is written between steps to flush L2.  The e2e figure runs
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
MODE_NAMES = {0x100: "block", 0x200: "graph", 0x300: "hostloop", 0x400: "persist"}


PRECISION_TEXT = {"fp64": "fp64 arithmetic and state",
                  "mixed": "fp32 per-slot arithmetic, fp64 state", "fp32": "fp32"}
DTYPES = {"fp64": "f64", "mixed": "f32", "fp32": "f32"}


def make_workload(name, precision="fp64"):
    """-> (list of Scene environments, description, batched?)"""
    p = PRECISION_TEXT[precision]
    if name == "batch256":
        return (scenes.env_batch(256, seed=0),
                f"256 uneven mass-spring envs (seed 0), SNH, {p}", True)
    if name.startswith("cantilever"):
        n = int(name[len("cantilever"):])
        return [scenes.cantilever(n)], f"cantilever {n}x{n // 10}x{n // 10} SNH, {p}", False
    if name == "massspring":
        return [scenes.mass_spring(11, 20)], f"mass-spring 11^3 cube + 1x1x20 column SNH, {p}", \
            False
    raise SystemExit(f"unknown workload {name}")


def sweep_bytes(s):
    """Algorithmic bytes of one sweep of one mesh: sum over solved vertices of
    B(v) = 44 + 104 k_v (fp32 storage, no reuse between vertices credited:
    44 B of per-vertex state -- x read and written, inertia target, lumped
    mass, adjacency offset -- and per incident tet 104 B: tet id, 4 vertex
    ids, Dm^-1, rest volume, (mu', lambda'), three neighbour positions)."""
    k = np.bincount(s.tets.reshape(-1), minlength=s.n_vertices)
    solved = s.active & (k > 0)
    return float((44 + 104 * k[solved]).sum()), int(solved.sum()), int(k[solved].sum())


def warm_stage_bytes(s):
    """Algorithmic bytes of the learned warm start's energy check of one mesh
    (the inertia guess and the full prediction compared in one pass over the
    mesh's tet list, fp32 storage like sweep_bytes): per tet with a solved
    vertex 176 B (4 vertex ids 16, Dm^-1 36, volume 4, (mu', lambda') 8, the
    four positions 48 and predictions 64), per solved vertex 44 B (position,
    inertia target, lumped mass, prediction).  The line search's further
    candidates (taken when the first raises the energy) are not counted."""
    k = np.bincount(s.tets.reshape(-1), minlength=s.n_vertices)
    solved = s.active & (k > 0)
    tets_solved = int(solved[s.tets].any(axis=1).sum())
    return float(176 * tets_solved + 44 * int(solved.sum()))


_REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
            ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))


class _NvmlSampler:
    """SM clock and clock-event reasons of one GPU every `period` seconds,
    read through NVML in a thread (read-only queries)."""

    def __init__(self, device, period=0.005):
        import threading

        import pynvml
        import torch
        self.nv = pynvml
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(device)
        try:
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(
                "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id))
        except Exception:
            self.h = pynvml.nvmlDeviceGetHandleByIndex(int(torch.device(device).index or 0))
        self.max = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        self.sm, self.bits, self.period = [], 0, period
        self.stop_ev = threading.Event()
        self.th = threading.Thread(target=self._run, daemon=True)
        self._sample()
        self.th.start()

    def _sample(self):
        self.sm.append(float(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)))
        self.bits |= int(self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))

    def _run(self):
        while not self.stop_ev.wait(self.period):
            self._sample()

    def stop(self):
        self.stop_ev.set()
        self.th.join(timeout=5)
        self._sample()
        self.nv.nvmlShutdown()
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": self.max,
                "reasons": sorted(n for n, b in _REASONS if self.bits & b),
                "samples": len(self.sm), "source": "nvml"}


def clocks_start(device=0):
    try:
        return _NvmlSampler(device)
    except Exception:
        pass
    try:
        return subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except Exception:
        return None


def clocks_stop(p, gpu_index):
    if p is None:
        return None
    if isinstance(p, _NvmlSampler):
        try:
            return p.stop()
        except Exception:
            return None
    p.terminate()
    try:
        out, _ = p.communicate(timeout=5)
    except Exception:
        p.kill()
        return None
    sm, mx, reasons = [], [], set()
    for line in out.strip().splitlines():
        c = [x.strip() for x in line.split(",")]
        if len(c) < 9 or c[0] != str(gpu_index):
            continue
        try:
            sm.append(float(c[1]))
            mx.append(float(c[2]))
        except ValueError:
            continue
        for (n, _), v in zip(_REASONS, c[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
            "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def sweep_histogram(iters):
    """Sweep counts of every (environment, step) pair in power-of-two bins:
    counts[i] holds the pairs with edges[i] <= sweeps < edges[i + 1]."""
    edges = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, MAX_ITER + 1]
    counts, _ = np.histogram(np.asarray(iters).reshape(-1), bins=edges)
    return {"edges": edges, "counts": counts.tolist()}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic_per_slot(kernel, workload):
    """DRAM bytes per (vertex, tet) slot visit that ncu measured for `kernel`
    on `workload` (summary committed under profiles/), or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.{workload}.md")
    try:
        for line in open(path):
            if line.strip().startswith("dram_bytes_per_slot_visit:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def concat(envs):
    """Concatenate environments into one mesh: the reference's own way of
    batching (examples/run_mass_spring_parallel.py:40-58)."""
    X, T, rho, E, nu, act = [], [], [], [], [], []
    off = 0
    for e in envs:
        X.append(e.vertices)
        T.append(e.tets + off)
        rho.append(e.density)
        E.append(e.youngs)
        nu.append(e.poisson)
        act.append(e.active)
        off += e.n_vertices
    return dict(initial_positions=np.concatenate(X), elements=np.concatenate(T),
                densities=np.concatenate(rho), youngs_modulus=np.concatenate(E),
                poissons_ratio=np.concatenate(nu), active_mask=np.concatenate(act))


def oracle_rate(envs, budget_s, max_steps, warmup=0, threads=None):
    """The FP64 oracle (OpenMP on all host threads, or `threads`) stepping
    `envs` as one concatenated mesh, as the reference batches; returns
    (env-sim-s per wall-s, steps, threads, seconds)."""
    from oracle import oracle
    n = threads or oracle.max_threads()
    oracle.set_threads(n)
    o = oracle.OracleSolver(**concat(envs), damping_coefficient=0.0, dx_tol=TOL,
                            max_iter=MAX_ITER, guarded=True)
    for _ in range(warmup):
        o.step(None, DT)
    t0 = time.perf_counter()
    k = 0
    while k < max_steps and (k == 0 or time.perf_counter() - t0 < budget_s):
        o.step(None, DT)
        k += 1
    el = time.perf_counter() - t0
    return len(envs) * k * DT / el, k, n, el


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def cpu_sample(envs, batched):
    return envs[:8] if batched else envs[:1]


def run_reference(args, envs, desc, batched):
    # a host-only run: no process group; under torchrun rank 0 alone times it
    # and the other ranks exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sample = cpu_sample(envs, batched)
    v, k, n, el = oracle_rate(sample, args.reference_budget_s, args.steps, warmup=args.warmup)
    what = (f"{len(sample)} of the {len(envs)} environments concatenated into one mesh "
            "(the reference's batching, one global convergence test)") if batched else \
        "the whole mesh"
    line = {"impl": "reference", "metric": "sim-s/wall-s", "value": v, "unit": "sim-s/wall-s",
            "n_gpus": args.gpus, "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * el / k,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "dt": DT, "tol": TOL, "max_iter": MAX_ITER},
            "cpu_baseline": {"value": v, "unit": "sim-s/wall-s", "cores": n, "kind": "port",
                             "sample": f"{k} whole steps of {what}; FP64 C restatement of the "
                                       "reference solver (warp-lang is not installable offline)"},
            "e2e": {"value": v, "unit": "sim-s/wall-s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def tuned_config(envs, batched, local, mode="auto", use=True, warm=False, precision="fp64"):
    """The autotuner's cached launch shape for this workload on this GPU
    (warpvbd_b200/data/autotune_b200.json or the user cache), or None.
    `warm`: the shape tuned with the learned warm start on (falls back to
    the plain shape)."""
    if not use or (not batched and mode != "auto"):
        return None
    from warpvbd_b200 import autotune
    dev = f"cuda:{local}"
    if batched:
        return ((autotune.cached_batched(envs, device=dev, warm=True, precision=precision)
                 if warm else None)
                or autotune.cached_batched(envs, device=dev, precision=precision))
    return autotune.cached_single(envs[0].solver_kwargs(), device=dev, precision=precision)


def make_solver(envs, batched, local, mode="auto", warm=None, tuned=None, precision="fp64",
                dx_tol=TOL, max_iter=MAX_ITER):
    if batched:
        from warpvbd_b200 import BatchedVBDSolver
        sol = BatchedVBDSolver(envs, dx_tol=dx_tol, max_iter=max_iter, device=f"cuda:{local}",
                               precision=precision, **(tuned or {}))
    else:
        from warpvbd_b200 import VBDSolver
        s = envs[0]
        shape = tuned or {"mode": mode}
        sol = VBDSolver(**s.solver_kwargs(), damping_coefficient=0.0, dx_tol=dx_tol,
                        max_iter=max_iter, device=f"cuda:{local}", precision=precision, **shape)
    if warm is not None:
        sol.set_warmstart(warm)
    return sol


def solver_for(args, envs, batched, local, warm, precision=None, dx_tol=TOL):
    """A solver of the workload with its tuned launch shape (and the tuned
    shape's description).  A tolerance other than the workload's (the
    accuracy reference) gets 20,000 sweeps at most."""
    precision = precision or args.precision
    tuned = tuned_config(envs, batched, local, args.mode, not args.no_tune, warm is not None,
                         precision)
    return make_solver(envs, batched, local, args.mode, warm, tuned, precision, dx_tol,
                       MAX_ITER if dx_tol == TOL else 20000), tuned


def warm_params(args, batched):
    """Trained warm-start model (committed file) for the batched workloads
    with --warmstart on."""
    if args.warmstart == "off" or not batched:
        return None
    from warpvbd_b200 import warmstart
    return warmstart.load()


def step_async(sol, batched):
    if batched:
        sol.step(DT, blocking=False)
    else:
        sol.step(sol.old_positions, DT, blocking=False)


def advance(sol, batched, steps):
    """Untimed steps (the lead-in to the timed window)."""
    for _ in range(steps):
        step_async(sol, batched)
        sol.sync()


def timed_steps(sol, batched, steps, warmup, local, flush, sample_clocks=False, detail=None):
    """Per-step CUDA-event times (ms) and per-step sweep counts.  `detail`
    (a dict) receives the step kernels' own CUDA-event times (the library
    records events around them on its stream) and the kernels launched."""
    import torch
    stream = torch.cuda.ExternalStream(sol.stream, device=local)
    advance(sol, batched, warmup)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    iters = []
    torch.cuda.synchronize()
    clk = clocks_start(local) if sample_clocks else None
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xFF)
        evs[k][0].record(stream)
        step_async(sol, batched)
        evs[k][1].record(stream)
        iters.append(np.array(sol.sync(), dtype=np.int64).reshape(-1))
        if detail is not None:
            inf = sol.info()
            detail.setdefault("kernel_ms", []).append(float(inf["last_step_kernel_ms"]))
            detail.setdefault("launches", []).append(int(inf["last_step_launches"]))
    torch.cuda.synchronize()
    clocks = clocks_stop(clk, local) if sample_clocks else None
    ms = np.array([a.elapsed_time(b) for a, b in evs])
    return ms, np.stack(iters), clocks


def tip_displacements(sol, envs):
    """Each environment's tip displacement (mean over its tip vertices of
    position minus rest position), [n_env][3]."""
    if len(envs) == 1 and not hasattr(sol, "env_slice"):
        x = sol.old_positions.numpy()
        e = envs[0]
        return ((x[e.tip] - e.vertices[e.tip]).mean(0))[None, :]
    x = sol.positions()
    out = np.empty((len(envs), 3))
    for i, e in enumerate(envs):
        xe = x[sol.env_slice(i)]
        out[i] = (xe[e.tip] - e.vertices[e.tip]).mean(0)
    return out


def tip_error(warm, plain, precision):
    """Tip error of the warm-started run against the plain run at the same
    tolerance (in fp64 the plain run is the FP64 oracle's trajectory to
    rounding): |d_warm - d_plain| at each checkpoint over the environment's
    largest plain tip displacement of all checkpoints.  warm / plain:
    [checkpoints][n_env][3]."""
    scale = np.linalg.norm(plain, axis=2).max(0)
    rel = np.linalg.norm(warm - plain, axis=2) / scale[None, :]
    return {"against": ("plain VBD in fp64 at the same tolerance (the FP64 oracle's "
                        "trajectory to rounding)" if precision == "fp64" else
                        f"plain VBD in {precision} at the same tolerance"),
            "normalised_by": "the environment's largest plain tip displacement",
            "max": float(rel.max()), "median": float(np.median(rel)),
            "max_by_checkpoint": [float(v) for v in rel.max(1)],
            "median_by_checkpoint": [float(v) for v in np.median(rel, 1)],
            "target": 1e-4, "within_target": bool(rel.max() <= 1e-4)}


def max_over_ranks(x, world, local):
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], device=f"cuda:{local}")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, envs, desc, batched):
    import torch
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    warm = warm_params(args, batched)
    sol, tuned = solver_for(args, envs, batched, local, warm)
    info = sol.info()
    advance(sol, batched, args.start_step)
    # the state at the start of the window, so that the end-to-end run below
    # covers the same steps
    snap = (sol.positions(), sol.velocities()) if batched else sol.get_state()
    if world > 1:
        torch.distributed.barrier()
    detail = {}
    ms, iters, clocks = timed_steps(sol, batched, args.steps, args.warmup, local, flush,
                                    sample_clocks=True, detail=detail)
    total_ms = max_over_ranks(float(ms.sum()), world, local)
    n_env = len(envs)
    value = world * n_env * args.steps * DT / (total_ms * 1e-3)

    # end to end through the public API: every step uploads the positions
    # from page-locked host memory and downloads the new ones into it.  The
    # run restarts from the window's first state and takes the same warm-up
    # and timed steps, so it covers the same part of the trajectory as
    # `value` (wall clock around the timed steps, max over ranks)
    n_vertices = sum(e.n_vertices for e in envs)
    e2e_steps = args.e2e_steps or args.steps
    xh = torch.empty((n_vertices, 3), dtype=torch.float64, pin_memory=True).numpy()
    sol.set_state(positions=snap[0], velocities=snap[1])
    xh[:] = snap[0]
    if world > 1:
        torch.distributed.barrier()
    if batched:
        # step(out=...) : the step kernels write each environment's positions
        # into the page-locked array as it finishes
        for k in range(args.warmup + e2e_steps):
            if k == args.warmup:
                t0 = time.perf_counter()
            sol.set_state(positions=xh)
            sol.step(DT, out=xh)
        e2e_s = time.perf_counter() - t0
    else:
        for k in range(args.warmup + e2e_steps):
            if k == args.warmup:
                t0 = time.perf_counter()
            sol.step(xh, DT).numpy(out=xh)
        e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world, local)
    e2e = world * n_env * e2e_steps * DT / e2e_s

    # roofline of the dominant kernel: algorithmic bytes of the sweeps it ran
    # (and of the warm start's energy check) over its own CUDA-event time
    per_env = [sweep_bytes(e) for e in envs]
    b_sweep = np.array([p[0] for p in per_env])
    slots = np.array([p[2] for p in per_env])
    solved = np.array([p[1] for p in per_env])
    b_warm = np.array([warm_stage_bytes(e) for e in envs]) if warm is not None else 0.0
    mode = MODE_NAMES[info["mode"]]
    alg_bytes = float((iters * b_sweep[None, :]).sum()) + args.steps * float(np.sum(b_warm))
    # the dominant kernel's own time: the library's events around the step
    # kernels (both tiers; without the warm-start feature / inference kernels)
    kernel_ms = float(np.sum(detail["kernel_ms"]))
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    kernel = {"block": "env_step_kernel", "persist": "persist_kernel"}.get(mode, "color_kernel")
    prof = f"{args.workload}.{args.precision}" + (".warm" if warm is not None else "")
    tps = profile_traffic_per_slot(kernel, prof)
    traffic = None if tps is None else tps * float((iters * slots[None, :]).sum()) / args.steps
    launches = int(np.sum(detail["launches"]))  # counted by the library, per step
    line = {"metric": "sim-s/wall-s", "value": value, "unit": "sim-s/wall-s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPES[args.precision], "data": "synthetic",
            "config": {"workload": desc, "n_env": n_env, "vertices": n_vertices,
                       "tets": int(sum(e.n_tets for e in envs)), "dt": DT, "tol": TOL,
                       "max_iter": MAX_ITER, "precision": args.precision,
                       "timed_window": f"steps {args.start_step + args.warmup + 1}-"
                                       f"{args.start_step + args.warmup + args.steps} "
                                       "of the trajectory from rest",
                       "mode": mode, "tpv": info["tpv"],
                       "block_threads": info["block_threads"],
                       "parallelism": f"replicas x{world}",
                       "warm_start": warm is not None, "cluster": info["cluster"],
                       "order_index": bool((tuned or {}).get("order_index", False)),
                       "autotuned": tuned is not None,
                       "tiered": bool((tuned or {}).get("tiered", False)),
                       "wide_tier": bool((tuned or {}).get("tiered", False)
                                         and (tuned or {}).get("wide_tier", True)),
                       "l2": "256 MiB written between timed steps"},
            "iters_per_step": {"hist": sweep_histogram(iters),
                               "mean": float(iters.mean()), "max": int(iters.max()),
                               "min": int(iters.min())},
            "vertex_updates_per_s": world * float((iters * solved[None, :]).sum())
            / (total_ms * 1e-3),
            "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes / args.steps,
                         "bytes_model": "B(v) = 44 + 104 k_v per vertex update, fp32 storage; "
                                        "warm-start check: 176 B per tet + 44 B per vertex",
                         "limiter": "issue and latency: the records and slots stay in L2 and "
                                    "the positions in shared memory, DRAM traffic is a small "
                                    "fraction of the algorithmic bytes (ncu summary in "
                                    "profiles/)" if mode == "block" else
                                    "latency: the per-colour dependency chain and grid "
                                    "barriers (ncu summary in profiles/)",
                         "kernel_ms_per_step": kernel_ms / args.steps},
            "e2e": {"value": e2e, "unit": "sim-s/wall-s",
                    "h2d_bytes_per_step": 24 * n_vertices,
                    "d2h_bytes_per_step": 24 * n_vertices,
                    "steps": e2e_steps,
                    "window": "the value's warm-up and timed steps, rerun from the window's "
                              "first state with host arrays in and out"},
            "gpu_launches": launches}
    if clocks:
        line["clocks"] = clocks
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = cpu_sample(envs, batched)
        v, k, n, el = oracle_rate(sample, args.cpu_budget_s, 50)
        line["cpu_baseline"] = {
            "value": v, "unit": "sim-s/wall-s", "cores": n, "kind": "port",
            "sample": f"{k} whole steps from rest of {len(sample)} environment(s) "
                      + ("concatenated into one mesh " if batched else "")
                      + f"({el:.1f} s), FP64 C oracle, OpenMP {n} threads"}
        # the reference's Warp CPU device runs its kernels on one thread: the
        # same oracle on one thread, one environment, a few seconds
        v1, k1, _, el1 = oracle_rate(sample[:1], min(5.0, args.cpu_budget_s), 50, threads=1)
        line["cpu_baseline"]["single_thread"] = {
            "value": v1, "sample": f"{k1} whole steps of 1 environment ({el1:.1f} s), 1 thread"}
    sol.close()
    if batched and not args.no_secondary:
        # the same batch with the learned warm start toggled (same window,
        # same timing method); every rank takes this path, so the collectives
        # match
        from warpvbd_b200 import warmstart
        other = None if warm is not None else warmstart.load()
        ps, _ = solver_for(args, envs, batched, local, other)
        advance(ps, batched, args.start_step)
        pms, pit, _ = timed_steps(ps, batched, args.steps, args.warmup, local, flush)
        pt = max_over_ranks(float(pms.sum()), world, local)
        pbytes = float((pit * b_sweep[None, :]).sum())
        if other is not None:
            pbytes += args.steps * float(np.sum([warm_stage_bytes(e) for e in envs]))
        pv = world * n_env * args.steps * DT / (pt * 1e-3)
        key = "warm_start_batched" if other is not None else "plain_batched"
        pinfo = ps.info()
        line[key] = {
            "value": pv, "ms_per_step": pt / args.steps,
            "iters_per_step": {"mean": float(pit.mean()), "max": int(pit.max()),
                               "hist": sweep_histogram(pit)},
            "roofline_frac": pbytes / (pt * 1e-3) / 1e9 / peak,
            "shape": {"tpv": pinfo["tpv"], "block_threads": pinfo["block_threads"],
                      "cluster": pinfo["cluster"]}}
        warm_v, plain_v = (pv, value) if other is not None else (value, pv)
        line["warm_start_speedup_vs_plain_batched"] = warm_v / plain_v
        ps.close()
    if rank == 0 and world == 1 and batched and not args.no_secondary:
        # plain VBD one environment at a time (single-environment solver), on a
        # sample of the batch: what the batch costs without batching
        t_seq, n_seq = 0.0, 0
        for env in envs[:16]:
            es = make_solver([env], False, local, precision=args.precision)
            ems, _, _ = timed_steps(es, False, 5, 3, local, flush)
            t_seq += float(ems.sum()) * 1e-3
            n_seq += 5
            es.close()
        line["plain_one_env_at_a_time"] = {
            "value": n_seq * DT / t_seq, "sample": "16 environments x 5 steps each, from rest"}
        # the workload's whole trajectory from rest, plain and warm-started,
        # every step device-timed
        from warpvbd_b200 import warmstart
        long, tips = {}, {}
        for name, model, tol in (("plain", None, TOL), ("warm_start", warmstart.load(), TOL),
                                 ("plain_tol_1e-9", None, 1e-9)):
            if tol != TOL and args.no_accuracy_run:
                continue
            ls, _ = solver_for(args, envs, batched, local, model, dx_tol=tol)
            # 100 steps at a time; each environment's tip displacement is
            # read (untimed) between the chunks
            chunks, tip = [], []
            for c0 in range(0, args.long_steps, 100):
                chunks.append(timed_steps(ls, batched, min(100, args.long_steps - c0), 0, local,
                                          flush))
                tip.append(tip_displacements(ls, envs))
            lms = np.concatenate([c[0] for c in chunks])
            lit = np.concatenate([c[1] for c in chunks])
            tips[name] = np.stack(tip)
            if tol != TOL:
                # the accuracy reference: untimed figures only
                long[name] = {"iters_per_step": {"mean": float(lit.mean()), "max": int(lit.max())},
                              "ms_per_step": float(lms.mean())}
                ls.close()
                continue
            long[name] = {"ms_per_step": float(lms.mean()),
                          "iters_per_step": {"mean": float(lit.mean()), "max": int(lit.max())},
                          "value": n_env * DT / (float(lms.mean()) * 1e-3),
                          "ms_per_step_by_100_steps": [
                              round(float(lms[i:i + 100].mean()), 4)
                              for i in range(0, args.long_steps, 100)]}
            ls.close()
        long["warm_start_speedup"] = (long["plain"]["ms_per_step"]
                                      / long["warm_start"]["ms_per_step"])
        long["warm_start_tip_error"] = tip_error(tips["warm_start"], tips["plain"],
                                                 args.precision)
        if "plain_tol_1e-9" in tips:
            # both forms against the same near-converged trajectory (plain
            # VBD at tol 1e-9): the accuracy each buys at tol 1e-7
            ref = tips["plain_tol_1e-9"]
            long["tip_error_vs_tol_1e-9"] = {
                name: {k: v for k, v in tip_error(tips[name], ref, args.precision).items()
                       if k not in ("against", "normalised_by", "target", "within_target")}
                for name in ("plain", "warm_start")}
            long["tip_error_vs_tol_1e-9"]["normalised_by"] = (
                "the environment's largest tip displacement in the tol-1e-9 run")
        line[f"batch_{args.long_steps}_steps"] = long
        if args.precision != "mixed":
            # the fp32-arithmetic mode on the same window, for comparison:
            # faster, but its trajectories drift from the fp64 ones
            ms_, _ = solver_for(args, envs, batched, local, warm, precision="mixed")
            advance(ms_, batched, args.start_step)
            mms, mit, _ = timed_steps(ms_, batched, args.steps, args.warmup, local, flush)
            line["mixed_precision_same_window"] = {
                "value": n_env * args.steps * DT / (float(mms.sum()) * 1e-3),
                "ms_per_step": float(mms.mean()), "iters_per_step": float(mit.mean()),
                "warm_start": warm is not None}
            ms_.close()
    if rank == 0 and world == 1 and batched and not args.no_secondary:
        # the plain single-mesh solver on the largest cantilever of the
        # resolution sweep, 320x32x32 (349,569 vertices; from rest)
        big = scenes.cantilever(320)
        bs, _ = solver_for(args, [big], False, local, None)
        bdet = {}
        bms, bit, _ = timed_steps(bs, False, 10, 3, local, flush, detail=bdet)
        bb, bsolved, _ = sweep_bytes(big)
        tb = float(bms.sum()) * 1e-3
        tbk = float(np.sum(bdet["kernel_ms"])) * 1e-3
        line["cantilever320"] = {
            "sim_s_per_wall_s": 10 * DT / tb, "ms_per_step": 1e3 * tb / 10,
            "iters_per_step": float(bit.mean()), "mode": MODE_NAMES[bs.info()["mode"]],
            "vertex_updates_per_s": bsolved * float(bit.sum()) / tb,
            "roofline_frac": bb * float(bit.sum()) / tbk / 1e9 / peak,
            "kernel_ms_per_step": 1e3 * tbk / 10, "steps": "4-13 from rest"}
        bs.close()
        # the plain single-mesh solver on the 160x16x16 cantilever (from rest)
        cant = scenes.cantilever(160)
        cs, _ = solver_for(args, [cant], False, local, None)
        cdet = {}
        cms, cit, _ = timed_steps(cs, False, args.secondary_steps, 3, local, flush, detail=cdet)
        cb, csolved, _ = sweep_bytes(cant)
        t = float(cms.sum()) * 1e-3
        tk = float(np.sum(cdet["kernel_ms"])) * 1e-3
        line["cantilever160"] = {
            "sim_s_per_wall_s": args.secondary_steps * DT / t,
            "ms_per_step": 1e3 * t / args.secondary_steps,
            "iters_per_step": float(cit.mean()), "mode": MODE_NAMES[cs.info()["mode"]],
            "vertex_updates_per_s": csolved * float(cit.sum()) / t,
            "roofline_frac": cb * float(cit.sum()) / tk / 1e9 / peak,
            "kernel_ms_per_step": 1e3 * tk / args.secondary_steps}
        # the same cantilever with the learned warm start (persistent mode)
        from warpvbd_b200 import warmstart
        ws_, _ = solver_for(args, [cant], False, local, warmstart.load())
        wdet = {}
        wms, wit, _ = timed_steps(ws_, False, args.secondary_steps, 3, local, flush, detail=wdet)
        tw = float(wms.sum()) * 1e-3
        ctip = tip_error(tip_displacements(ws_, [cant])[None], tip_displacements(cs, [cant])[None],
                         args.precision)
        line["cantilever160_warm_start"] = {
            "tip_error_vs_plain": {k: ctip[k] for k in ("against", "max", "target")},
            "sim_s_per_wall_s": args.secondary_steps * DT / tw,
            "ms_per_step": 1e3 * tw / args.secondary_steps,
            "iters_per_step": float(wit.mean()),
            "kernel_ms_per_step": float(np.mean(wdet["kernel_ms"])),
            "speedup_vs_plain": t / tw}
        ws_.close()
        cs.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch256")
    ap.add_argument("--mode", default="auto",
                    choices=["auto", "block", "graph", "hostloop", "persist"])
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="timed end-to-end steps (0 = --steps)")
    ap.add_argument("--secondary-steps", type=int, default=30)
    ap.add_argument("--long-steps", type=int, default=1000,
                    help="steps of the whole-trajectory plain / warm-started batch comparison")
    ap.add_argument("--no-accuracy-run", action="store_true",
                    help="skip the tol-1e-9 reference trajectory of the whole-trajectory "
                         "comparison (about 22 s on B200)")
    ap.add_argument("--start-step", type=int, default=500,
                    help="untimed steps from rest before the warm-up and timed steps")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "fp32"])
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--reference-budget-s", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="ignore the autotuner's cached launch shapes (use the built-in defaults)")
    ap.add_argument("--warmstart", default="on", choices=["off", "on"],
                    help="the headline batched run starts steps from the trained network "
                         "(on: the metric's warm-start + batched form); the other setting is "
                         "timed beside it as plain_batched / warm_start_batched")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    envs, desc, batched = make_workload(args.workload, args.precision)
    if args.impl == "reference":
        run_reference(args, envs, desc, batched)
    else:
        run_ours(args, envs, desc, batched)


if __name__ == "__main__":
    main()
