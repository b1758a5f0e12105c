"""Environment sharding across ranks (CPU): the balanced partition, and a
world-size-2 gloo job whose ranks step their own shares with a stand-in
solver and gather positions and sweep counts to rank 0 in the original
order."""
import os
import socket

import numpy as np
import pytest

from warpvbd_b200 import distributed, scenes


def test_partition_covers_every_environment_once_and_balances():
    rng = np.random.default_rng(0)
    w = rng.uniform(1.0, 10.0, size=101)
    for n in (1, 2, 3, 8):
        parts = distributed.partition(w, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(101))
        loads = [w[p].sum() for p in parts]
        assert max(loads) - min(loads) <= w.max()   # greedy bound
    assert distributed.partition([5.0, 1.0], 4)[2:] == [[], []]


def test_env_weights_follow_the_mesh():
    envs = scenes.env_batch(6, seed=2)
    w = distributed.env_weights(envs)
    assert np.all(w > 0)
    sizes = np.array([e.n_vertices for e in envs])
    assert np.corrcoef(w, sizes)[0, 1] > 0.9


class _FakeSolver:
    """Stand-in for BatchedVBDSolver: environment j of the shard moves by
    (step count) x (its vertex count) along x; sweeps = vertex count."""

    def __init__(self, envs):
        self.envs = envs
        self.off = np.cumsum([0] + [e.n_vertices for e in envs])
        self.x = np.concatenate([e.vertices for e in envs]).copy()

    def step(self, dt):
        for j, e in enumerate(self.envs):
            self.x[self.off[j]:self.off[j + 1], 0] += e.n_vertices
        return np.array([e.n_vertices for e in self.envs])

    def positions(self):
        return self.x.copy()

    def env_slice(self, j):
        return slice(self.off[j], self.off[j + 1])


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        envs = scenes.env_batch(7, seed=5)
        shard = distributed.ShardedBatch(envs, solver_factory=lambda es: _FakeSolver(es))
        for _ in range(3):
            its = shard.step(1e-3)
        x = shard.gather_positions(0)
        it = shard.gather_iterations(its, 0)
        if rank == 0:
            ok = all(np.allclose(x[i][:, 0], e.vertices[:, 0] + 3 * e.n_vertices)
                     and np.allclose(x[i][:, 1:], e.vertices[:, 1:]) for i, e in enumerate(envs))
            ok = ok and np.array_equal(it, [e.n_vertices for e in envs])
            q.put(("ok" if ok else "mismatch", len(shard.mine)))
        else:
            assert x is None and it is None
            q.put(("rank1", len(shard.mine)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_job_gathers_in_original_order():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    tags = dict(res)
    assert tags.get("ok") is not None, res
    assert tags["ok"] + tags["rank1"] == 7 and tags["ok"] > 0 and tags["rank1"] > 0
