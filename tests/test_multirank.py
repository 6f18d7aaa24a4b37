"""The N>1 host path on CPU: world_size-2 gloo ranks shard a batch, transform
their slices, reduce the time with MAX and gather the results.

The per-rank transform here is the oracle (this is a CPU test of the sharding,
reduction and gather logic); on GPUs each rank runs its slice through the CUDA
library instead and nothing else changes.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fft3d_b200.dist import shard_range


def test_shard_range_partitions():
    for n in (0, 1, 2, 7, 2048, 4097):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            cover = []
            for s, c in spans:
                cover.extend(range(s, s + c))
            assert cover == list(range(n))
            counts = [c for _, c in spans]
            assert max(counts) - min(counts) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, shape, q):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "opt-fft_b200"))
    import oracle
    from fft3d_b200.dist import gather_volumes, max_over_ranks, shard_range as sr
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(77)
        x = rng.uniform(-1, 1, (n,) + shape) + 1j * rng.uniform(-1, 1, (n,) + shape)
        s, c = sr(n, rank, world)
        local = oracle.fft3d(x[s:s + c], nthreads=1) if c else np.zeros((0,) + shape, complex)
        t = max_over_ranks(0.5 + rank, dist)
        full = gather_volumes(torch.from_numpy(np.ascontiguousarray(local)), n, dist).numpy()
        ok = np.array_equal(full, oracle.fft3d(x, nthreads=1)) and t == 0.5 + world - 1
        q.put((rank, bool(ok), c))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [9, 1])
def test_two_rank_shard_gather(n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    shape = (8, 8, 8)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, shape, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert all(ok for _, ok, _ in res), res
    assert sum(c for _, _, c in res) == n
    assert all(p.exitcode == 0 for p in procs)
