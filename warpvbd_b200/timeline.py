"""Step timeline of a batched solve: where each thread block of a step ran.

    python -m warpvbd_b200.timeline [--envs 256] [--seed 0] [--steps 24] [--skip 4]
                                    [--warm] [--out timeline.json]

Steps the seeded batch of uneven mass-spring environments (the benchmark batch:
``scenes.env_batch(n, seed)``) with the autotuned launch shape, records every
block of every step (``BatchedVBDSolver.set_trace``) and prints, per step, the
step-kernel time, the number of blocks and how full the device's block slots
were, then the blocks that ended last (the environments that set the step
time), and the cost per slot visit of single-block and split environments.
"""
import argparse
import json

import numpy as np


def blocks_per_sm(tl):
    """Largest number of blocks seen running at once on one SM."""
    best = 0
    for sm in np.unique(tl["sm"]):
        on = tl["sm"] == sm
        ev = sorted([(int(t), 1) for t in tl["start_ns"][on]] +
                    [(int(t), -1) for t in tl["end_ns"][on]])
        cur = 0
        for _, d in ev:
            cur += d
            best = max(best, cur)
    return best


def busy_fraction(tl, n_slots):
    """Block time of the step / (block slots x step length)."""
    span = float(tl["end_ns"].max()) if len(tl["end_ns"]) else 0.0
    work = float((tl["end_ns"] - tl["start_ns"]).sum())
    return work / (n_slots * span) if span > 0 else 0.0


def summarize(steps, env_slots, n_slots):
    """Per-step rows and the per-class cost (ns per slot visit per block)."""
    rows, cost = [], {}
    for st in steps:
        tl = st["timeline"]
        it = np.asarray(st["iters"])
        rows.append({"kernel_ms": st["kernel_ms"], "blocks": int(len(tl["env"])),
                     "split_blocks": int((tl["launch"] == 0).sum()),
                     "busy": busy_fraction(tl, n_slots),
                     "last": [int(e) for e in tl["env"][np.argsort(-tl["end_ns"])[:3]]],
                     "sweeps_max": int(it.max()), "sweeps_mean": float(it.mean())})
        for i in range(len(tl["env"])):
            e = int(tl["env"][i])
            ranks = int((tl["env"] == e).sum())
            cls = "single" if ranks == 1 else f"split{ranks}"
            c = cost.setdefault(cls, [0.0, 0.0])
            c[0] += float(tl["end_ns"][i] - tl["start_ns"][i])
            c[1] += env_slots[e] * max(int(it[e]), 1) / ranks
    return rows, {k: v[0] / v[1] for k, v in cost.items() if v[1] > 0}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--envs", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--skip", type=int, default=4, help="untraced steps first")
    ap.add_argument("--warm", action="store_true", help="with the learned warm start")
    ap.add_argument("--out", default=None, help="write every block's record as JSON")
    a = ap.parse_args(argv)

    import torch

    from . import autotune, scenes, warmstart
    from .batched import BatchedVBDSolver
    envs = scenes.env_batch(a.envs, seed=a.seed)
    shape = ((autotune.cached_batched(envs, warm=True) if a.warm else None)
             or autotune.cached_batched(envs) or {})
    sol = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000, **shape)
    if a.warm:
        sol.set_warmstart(warmstart.load())
    slots = np.array([4.0 * e.n_tets for e in envs])
    n_sms = torch.cuda.get_device_properties(0).multi_processor_count
    for _ in range(a.skip):
        sol.step(1e-3)
    sol.set_trace(True)
    steps = []
    for _ in range(a.steps):
        it = sol.step(1e-3)
        steps.append({"iters": it, "kernel_ms": sol.info()["last_step_kernel_ms"],
                      "timeline": sol.timeline()})
    sol.close()
    per_sm = max(blocks_per_sm(s["timeline"]) for s in steps)
    n_slots = n_sms * per_sm
    rows, cost = summarize(steps, slots, n_slots)
    print(f"shape {shape}, warm start {a.warm}, {a.envs} environments, "
          f"{n_sms} SMs x {per_sm} resident block(s)")
    for k, r in enumerate(rows):
        print(f"step {k:3d}: {r['kernel_ms']:.3f} ms, {r['blocks']} blocks "
              f"({r['split_blocks']} split), slots busy {r['busy']:.2f}, sweeps mean "
              f"{r['sweeps_mean']:.1f} max {r['sweeps_max']}, last to end: envs {r['last']}")
    for k, v in sorted(cost.items()):
        print(f"{k}: {v:.2f} ns per slot visit per block")
    if a.out:
        with open(a.out, "w") as f:
            json.dump({"shape": shape, "warm": a.warm, "env_slots": slots.tolist(),
                       "steps": [{"iters": s["iters"].tolist(), "kernel_ms": s["kernel_ms"],
                                  **{k: v.tolist() for k, v in s["timeline"].items()}}
                                 for s in steps]}, f)
    return rows, cost


if __name__ == "__main__":
    main()
