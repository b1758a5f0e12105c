"""ShardedBatch on one GPU (world size 1, gloo process group): the same
environments stepped through the shard and directly through
BatchedVBDSolver must give identical positions."""
import os
import socket

import numpy as np
import pytest

from warpvbd_b200 import scenes

pytestmark = pytest.mark.gpu


def test_sharded_batch_world_one_matches_batched_solver():
    import torch.distributed as dist
    from warpvbd_b200 import BatchedVBDSolver
    from warpvbd_b200.distributed import ShardedBatch
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        envs = scenes.env_batch(5, seed=8)
        shard = ShardedBatch(envs, dx_tol=1e-7, max_iter=1000)
        ref = BatchedVBDSolver(envs, dx_tol=1e-7, max_iter=1000)
        for _ in range(5):
            a = shard.step(1e-3)
            b = ref.step(1e-3)
            assert np.array_equal(a, b)
        x = shard.gather_positions(0)
        xr = ref.positions()
        for i in range(len(envs)):
            assert np.array_equal(x[i], xr[ref.env_slice(i)])
    finally:
        dist.destroy_process_group()
