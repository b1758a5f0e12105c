"""Batched environments over several GPUs: one process per GPU, environments
sharded across the processes, no collective on the step path.

Environments are independent, so each rank steps its own share with its own
BatchedVBDSolver and nothing crosses the interconnect while stepping; results
are gathered only when asked (positions or sweep counts to one rank, with
torch.distributed object collectives).  The share of each rank is balanced by
the environments' algorithmic bytes per sweep (sum over solved vertices of
44 + 104 x valence), the measure the step's cost scales with, by a greedy
longest-first assignment.

    torch.distributed.init_process_group("nccl")       # the caller's job
    shard = ShardedBatch(envs, dx_tol=1e-7, max_iter=1000)
    for _ in range(steps):
        shard.step(1e-3)
    x = shard.gather_positions(dst=0)                  # list per environment on rank 0

A single mesh does not shard this way (its colours would need a halo
exchange per colour); it runs on one GPU.
"""
import heapq

import numpy as np


def env_weights(envs):
    """Algorithmic bytes of one sweep of each environment."""
    out = []
    for e in envs:
        k = np.bincount(np.asarray(e.tets).reshape(-1), minlength=e.n_vertices)
        solved = np.asarray(e.active, bool) & (k > 0)
        out.append(float((44 + 104 * k[solved]).sum()))
    return np.asarray(out)


def partition(weights, n_parts):
    """Longest-first greedy: environment indices per part (each list in
    ascending order), every index exactly once, parts balanced by weight."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    w = np.asarray(weights, np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    heap = [(0.0, p) for p in range(n_parts)]
    heapq.heapify(heap)
    parts = [[] for _ in range(n_parts)]
    for i in order:
        load, p = heapq.heappop(heap)
        parts[p].append(i)
        heapq.heappush(heap, (load + w[i], p))
    return [sorted(p) for p in parts]


class ShardedBatch:
    """This rank's share of a batch of environments.  `solver_factory(envs,
    **solver_kwargs)` builds the local solver (default: BatchedVBDSolver on
    cuda:LOCAL_RANK); it must offer step(dt) -> sweeps per environment,
    positions() -> [V, 3] and env_slice(i)."""

    def __init__(self, envs, *, solver_factory=None, group=None, **solver_kwargs):
        import os

        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.n_env = len(envs)
        self.parts = partition(env_weights(envs), self.world)
        self.mine = self.parts[self.rank]
        if solver_factory is None:
            from .batched import BatchedVBDSolver
            local = int(os.environ.get("LOCAL_RANK", "0"))
            solver_kwargs.setdefault("device", f"cuda:{local}")
            solver_factory = BatchedVBDSolver
        self.solver = (solver_factory([envs[i] for i in self.mine], **solver_kwargs)
                       if self.mine else None)

    def step(self, dt):
        """One step of this rank's environments (no communication); returns
        their sweep counts (empty on a rank without environments)."""
        if self.solver is None:
            return np.zeros(0, np.int32)
        return np.asarray(self.solver.step(dt))

    def _gather(self, local, dst):
        out = [None] * self.world if self.rank == dst else None
        self.dist.gather_object(local, out, dst=dst, group=self.group)
        return out

    def gather_positions(self, dst=0):
        """Positions of every environment, in the original order, on rank
        `dst` (None on the others)."""
        local = []
        if self.solver is not None:
            x = self.solver.positions()
            local = [x[self.solver.env_slice(j)] for j in range(len(self.mine))]
        got = self._gather(local, dst)
        if got is None:
            return None
        res = [None] * self.n_env
        for part, arrs in zip(self.parts, got):
            for i, a in zip(part, arrs):
                res[i] = a
        return res

    def gather_iterations(self, local_iters, dst=0):
        """Per-environment sweep counts of the last step, original order, on
        rank `dst`."""
        got = self._gather(np.asarray(local_iters).tolist(), dst)
        if got is None:
            return None
        res = np.zeros(self.n_env, np.int64)
        for part, its in zip(self.parts, got):
            res[part] = its
        return res


__all__ = ["env_weights", "partition", "ShardedBatch"]
