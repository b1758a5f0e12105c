"""Launch-shape autotuner for the VBD solvers (not part of the reference).

The same mesh runs fastest under different schedules depending on its size
and shape.  Measured on a B200 (per sweep, cantilever meshes):

- up to a few hundred vertices, one thread block holding the whole mesh in
  shared memory (block mode) wins;
- at a few thousand, block mode wins only when the mesh is spread over a
  thread-block cluster;
- beyond that, one cooperative launch with grid barriers (persistent mode)
  or per-colour kernels in a graph (graph mode) is faster, and which lanes
  per vertex are best changes again.

The autotuner measures instead of guessing.  For one mesh (or one batch of
environments) it builds a solver per candidate launch shape, times a few
steps from the rest state with CUDA events on the solver's stream, and keeps
the fastest.

- Searched parameters: the mode; lanes per vertex (tpv); threads per block;
  the cluster size (block mode); and the vertex order inside a colour
  (by valence, or by index).
- Search method: coordinate descent inside each mode family, then the best
  family.
- Cache: results are kept in a JSON file keyed by a hash of the mesh, the
  material, the precision and the GPU name, so a mesh is tuned once per
  GPU type.

    cfg = autotune.tune_single(scene.solver_kwargs())       # -> dict of kwargs
    solver = VBDSolver(**scene.solver_kwargs(), **cfg)
    # or simply
    solver = VBDSolver(**scene.solver_kwargs(), tune=True)

Cache location: `cache_path` argument, else $WARPVBD_B200_TUNE_CACHE, else
~/.cache/warpvbd_b200/autotune.json.  The committed file
warpvbd_b200/data/autotune_b200.json holds results measured on B200 for the
benchmark workloads and is consulted first (read-only).
"""
import hashlib
import json
import math
import os
import time

import numpy as np

PACKAGE_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                             "autotune_b200.json")

# Candidate values per parameter, per mode family.
SINGLE_SPACE = {
    "block": {"tpv": [2, 4, 8, 16], "block_threads": [256, 512, 128],
              "cluster": [1, 2, 4, 8, 16], "order_index": [False, True]},
    "persist": {"tpv": [4, 2, 8, 16], "block_threads": [256, 512, 128],
                "order_index": [False, True]},
    "graph": {"tpv": [4, 2, 8, 16], "order_index": [False, True]},
}
BATCH_SPACE = {
    "block": {"tiered": [True, False], "wide_tier": [True, False],
              "cluster": [4, 8, 2, 16], "tpv": [4, 2, 8],
              "block_threads": [256, 128, 512], "order_index": [False, True]},
}
# Shared memory a block-mode step may use (bytes), and per vertex.
BLOCK_SMEM_LIMIT = 227 * 1024 - 2048
STATE_BYTES = {"fp32": 12, "mixed": 24, "fp64": 24}


def default_cache_path():
    p = os.environ.get("WARPVBD_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "warpvbd_b200", "autotune.json")


# ---------------------------------------------------------------------------
# Search (independent of the GPU; `evaluate` returns a cost, lower is better,
# math.inf for a candidate that cannot be built)
# ---------------------------------------------------------------------------
def coordinate_descent(space, evaluate, start=None, passes=2):
    """Minimise evaluate(config) over the product of `space` (dict name ->
    candidate values), one parameter at a time, each pass holding the others
    at the best so far.  Every distinct config is evaluated at most once.
    Returns (best_config, best_cost, log) with log = [(config, cost), ...]."""
    names = list(space)
    cur = dict(start) if start else {n: space[n][0] for n in names}
    seen = {}
    log = []

    def cost(cfg):
        key = tuple(sorted(cfg.items()))
        if key not in seen:
            c = evaluate(dict(cfg))
            seen[key] = c
            log.append((dict(cfg), c))
        return seen[key]

    best = cost(cur)
    for _ in range(passes):
        improved = False
        for n in names:
            for v in space[n]:
                if v == cur[n]:
                    continue
                cand = dict(cur, **{n: v})
                c = cost(cand)
                if c < best:
                    best, cur, improved = c, cand, True
        if not improved:
            break
    return cur, best, log


def search_families(spaces, evaluate, starts=None, passes=2):
    """coordinate_descent inside every mode family of `spaces` (dict mode ->
    space); returns (best config incl. "mode", cost, log)."""
    best, best_c, log = None, math.inf, []
    for mode, space in spaces.items():
        ev = lambda cfg, mode=mode: evaluate(dict(cfg, mode=mode))
        cfg, c, lg = coordinate_descent(space, ev, (starts or {}).get(mode), passes)
        log += [(dict(k, mode=mode), v) for k, v in lg]
        if c < best_c:
            best, best_c = dict(cfg, mode=mode), c
    return best, best_c, log


# ---------------------------------------------------------------------------
# Keys and cache
# ---------------------------------------------------------------------------
def _device_name(device):
    import torch
    idx = torch.device(device).index or 0
    return torch.cuda.get_device_name(idx)


def mesh_key(kind, tets, vertices, offsets, material, precision, device_name):
    h = hashlib.sha1()
    for a in (tets, vertices, offsets):
        if a is not None:
            a = np.ascontiguousarray(a)
            h.update(str(a.dtype).encode() + str(a.shape).encode())
            h.update(a.tobytes())
    h.update(f"{kind}|{material}|{precision}|{device_name}".encode())
    return h.hexdigest()


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(key, cache_path=None):
    """Cached configuration for `key`: the user cache, then the committed table."""
    for p in (cache_path or default_cache_path(), PACKAGE_TABLE):
        ent = _load(p).get(key)
        if ent:
            return ent["config"]
    return None


def store(key, config, info, cache_path=None):
    p = cache_path or default_cache_path()
    d = _load(p)
    d[key] = {"config": config, **info}
    os.makedirs(os.path.dirname(os.path.abspath(p)), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


# ---------------------------------------------------------------------------
# Measurement on the GPU
# ---------------------------------------------------------------------------
def _time_solver(sol, step, steps, warmup, batched):
    """(ms per sweep for one mesh, ms per step for a batch) over `steps`
    steps after `warmup`, with CUDA events on the solver's stream."""
    import torch
    for _ in range(warmup):
        step()
        sol.sync()
    dev = torch.device(sol.device) if isinstance(sol.device, str) else sol.device
    st = torch.cuda.ExternalStream(sol.stream, device=dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sweeps = 0
    torch.cuda.synchronize(dev)
    a.record(st)
    for _ in range(steps):
        step()
        it = sol.sync()
        sweeps += int(np.max(it))
    b.record(st)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b)
    return ms / steps if batched else ms / max(1, sweeps)


def _fits_block(n_vertices, precision):
    return n_vertices * STATE_BYTES[precision] <= BLOCK_SMEM_LIMIT


def tune_single(solver_kwargs, *, material="snh", precision="fp64", device="cuda",
                damping_coefficient=0.0, dt=1e-3, dx_tol=1e-7, max_iter=1000, steps=4, warmup=2,
                spaces=None, cache_path=None, refresh=False, verbose=False):
    """Fastest launch shape for one mesh: a dict of VBDSolver keyword
    arguments (mode, tpv, block_threads, cluster, order_index).
    `solver_kwargs` holds the mesh arguments of VBDSolver (initial_positions,
    elements, densities, youngs_modulus, poissons_ratio, active_mask)."""
    from .vbd_solver import VBDSolver
    kw = {k: v for k, v in solver_kwargs.items()
          if k not in ("damping_coefficient", "dx_tol", "max_iter", "device")}
    X = np.asarray(kw["initial_positions"], np.float64)
    T = np.asarray(kw["elements"], np.int32)
    name = _device_name(device)
    key = mesh_key("single", T, X, None, material, precision, name)
    if not refresh:
        hit = lookup(key, cache_path)
        if hit is not None:
            return hit
    if spaces is None:
        spaces = {m: s for m, s in SINGLE_SPACE.items()
                  if m != "block" or _fits_block(X.shape[0], precision)}

    def evaluate(cfg):
        mode = cfg["mode"]
        args = dict(mode=mode, tpv=cfg.get("tpv", 0), block_threads=cfg.get("block_threads", 0),
                    cluster=cfg.get("cluster", 0), order_index=cfg.get("order_index", False))
        try:
            sol = VBDSolver(**kw, damping_coefficient=damping_coefficient, dx_tol=dx_tol,
                            max_iter=max_iter, device=device, material=material,
                            precision=precision, **args)
        except Exception as e:  # a shape this mesh / device cannot run
            if verbose:
                print("skip", cfg, str(e)[:80])
            return math.inf
        try:
            c = _time_solver(sol, lambda: sol.step(sol.old_positions, dt, blocking=False),
                             steps, warmup, False)
        finally:
            sol.close()
        if verbose:
            print(f"{cfg}: {1e3 * c:.2f} us/sweep", flush=True)
        return c

    t0 = time.perf_counter()
    best, cost, log = search_families(spaces, evaluate)
    cfg = _kwargs(best)
    store(key, cfg, {"ms_per_sweep": cost, "device": name, "evaluated": len(log),
                     "tune_s": round(time.perf_counter() - t0, 1),
                     "n_vertices": int(X.shape[0]), "n_tets": int(T.shape[0])}, cache_path)
    return cfg


def tune_batched(envs, *, material="snh", precision="fp64", device="cuda", dt=1e-3,
                 dx_tol=1e-7, max_iter=1000, steps=12, warmup=300, spaces=None, cache_path=None,
                 refresh=False, verbose=False, warm=None):
    """Fastest launch shape for a batch of environments: a dict of
    BatchedVBDSolver keyword arguments (tpv, block_threads, cluster,
    order_index, tiered, wide_tier).  Each candidate runs `warmup` untimed
    and `steps` timed steps from rest: the sweep counts of a batch grow over
    its first few hundred steps as the motion develops and become uneven
    across environments, so a window at rest favours the wrong shape (the
    default times steps 301-312).
    With `warm` (a warm-start model, see warpvbd_b200.warmstart)
    the candidates are timed with the learned warm start on, and the result
    is cached under its own key: the warm-started sweep counts are far more
    uneven across environments, which favours other shapes."""
    from .batched import BatchedVBDSolver

    def get(env, key, attr):
        return env[key] if isinstance(env, dict) else getattr(env, attr)
    Xs = [np.asarray(get(e, "initial_positions", "vertices"), np.float64).reshape(-1, 3)
          for e in envs]
    tets = np.concatenate([np.asarray(get(e, "elements", "tets"), np.int32).reshape(-1)
                           for e in envs])
    verts = np.concatenate([x.reshape(-1) for x in Xs])
    offs = np.cumsum([0] + [x.shape[0] for x in Xs]).astype(np.int64)
    name = _device_name(device)
    key = mesh_key("batched-warm" if warm is not None else "batched", tets, verts, offs,
                   material, precision, name)
    if not refresh:
        hit = lookup(key, cache_path)
        if hit is not None:
            return hit
    spaces = spaces or BATCH_SPACE

    def evaluate(cfg):
        args = {k: cfg[k] for k in ("tpv", "block_threads", "cluster", "order_index", "tiered",
                                    "wide_tier") if k in cfg}
        try:
            sol = BatchedVBDSolver(envs, dx_tol=dx_tol, max_iter=max_iter, device=device,
                                   material=material, precision=precision, **args)
            if warm is not None:
                sol.set_warmstart(warm)
        except Exception as e:
            if verbose:
                print("skip", cfg, str(e)[:80])
            return math.inf
        try:
            c = _time_solver(sol, lambda: sol.step(dt, blocking=False), steps, warmup, True)
        finally:
            sol.close()
        if verbose:
            print(f"{cfg}: {c:.3f} ms/step", flush=True)
        return c

    t0 = time.perf_counter()
    best, cost, log = search_families(spaces, evaluate)
    cfg = {k: v for k, v in _kwargs(best).items() if k != "mode"}
    cfg["tiered"] = bool(best.get("tiered", False))
    cfg["wide_tier"] = cfg["tiered"] and bool(best.get("wide_tier", True))
    store(key, cfg, {"ms_per_step": cost, "device": name, "evaluated": len(log),
                     "tune_s": round(time.perf_counter() - t0, 1), "n_env": len(envs),
                     "n_vertices": int(offs[-1])}, cache_path)
    return cfg


def _kwargs(cfg):
    out = {"mode": cfg["mode"], "tpv": int(cfg.get("tpv", 0)),
           "block_threads": int(cfg.get("block_threads", 0)),
           "cluster": int(cfg.get("cluster", 0)), "order_index": bool(cfg.get("order_index", False))}
    if out["mode"] == "graph":
        out["block_threads"] = 0
    return out


def cached_single(solver_kwargs, *, material="snh", precision="fp64", device="cuda",
                  cache_path=None):
    """The cached configuration of a mesh (user cache, then the committed
    table), or None: nothing is measured."""
    X = np.asarray(solver_kwargs["initial_positions"], np.float64)
    T = np.asarray(solver_kwargs["elements"], np.int32)
    return lookup(mesh_key("single", T, X, None, material, precision, _device_name(device)),
                  cache_path)


def cached_batched(envs, *, material="snh", precision="fp64", device="cuda", cache_path=None,
                   warm=False):
    """The cached configuration of a batch (`warm`: tuned with the learned
    warm start on), or None: nothing is measured."""
    Xs = [np.asarray(e.vertices, np.float64).reshape(-1, 3) for e in envs]
    tets = np.concatenate([np.asarray(e.tets, np.int32).reshape(-1) for e in envs])
    verts = np.concatenate([x.reshape(-1) for x in Xs])
    offs = np.cumsum([0] + [x.shape[0] for x in Xs]).astype(np.int64)
    return lookup(mesh_key("batched-warm" if warm else "batched", tets, verts, offs, material,
                           precision, _device_name(device)), cache_path)


def benchmark_workload(name):
    """The benchmark workloads by name: batch256 (256 uneven mass-spring
    environments, seed 0), cantilever20/40/80/160/320, massspring.
    Returns (list of scenes, batched?)."""
    from . import scenes
    if name == "batch256":
        return scenes.env_batch(256, seed=0), True
    if name.startswith("cantilever"):
        return [scenes.cantilever(int(name[len("cantilever"):]))], False
    if name == "massspring":
        return [scenes.mass_spring(11, 20)], False
    raise ValueError(f"unknown workload {name}")


def main(argv=None):
    """python -m warpvbd_b200.autotune [--out PATH] [--refresh] WORKLOAD ...
    tunes the named benchmark workloads on this GPU into the cache at PATH."""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("workloads", nargs="+")
    ap.add_argument("--out", default=None, help="cache file (default: the user cache)")
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--refresh", action="store_true")
    ap.add_argument("--warm", action="store_true",
                    help="batched workloads: tune with the committed warm-start model on")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    out = {}
    for w in a.workloads:
        envs, batched = benchmark_workload(w)
        t0 = time.perf_counter()
        if batched:
            warm = None
            if a.warm:
                from . import warmstart
                warm = warmstart.load()
            cfg = tune_batched(envs, precision=a.precision, cache_path=a.out, refresh=a.refresh,
                               verbose=a.verbose, warm=warm)
        else:
            cfg = tune_single(envs[0].solver_kwargs(), precision=a.precision, cache_path=a.out,
                              refresh=a.refresh, verbose=a.verbose)
        out[w] = dict(cfg, tune_s=round(time.perf_counter() - t0, 1))
        print(w, json.dumps(out[w]), flush=True)
    return out


__all__ = ["tune_single", "tune_batched", "cached_single", "cached_batched",
           "benchmark_workload", "coordinate_descent", "search_families", "lookup",
           "store", "mesh_key", "default_cache_path", "PACKAGE_TABLE"]


if __name__ == "__main__":
    main()
