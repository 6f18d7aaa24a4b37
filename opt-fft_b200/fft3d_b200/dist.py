"""Multi-GPU batch sharding: one process per GPU, no collective on the data path.

Volumes are independent (the reference's multi-GPU floor is exactly this split,
bench/mgpu/impl_1/baseline_mgpu.cu:1-9), so a global batch is cut into one
contiguous, balanced slice per rank and each rank transforms its slice on its own
GPU.  Collectives appear only outside the transform: the max-over-ranks of a
timing and an optional gather of results for checking.

    from fft3d_b200.dist import ShardedPlan
    sp = ShardedPlan((17, 17, 17), global_batch, rank, world)
    sp.plan.execute(d_in_local, d_out_local, stream)   # this rank's sp.count volumes
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int):
    """(start, count) of rank's contiguous slice of n volumes; counts differ by <= 1."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request n={n} rank={rank} world={world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, dist, device=None) -> float:
    """All-reduce MAX of a scalar (the job time is the slowest rank's)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_volumes(local, n_total: int, dist):
    """All-gather the ranks' result slices (torch tensors, batch first) into the
    full batch on every rank.  Slices may differ in length by one volume."""
    import torch
    world = dist.get_world_size()
    counts = [shard_range(n_total, r, world)[1] for r in range(world)]
    m = max(counts) if counts else 0
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)


class ShardedPlan:
    """The plan for this rank's slice of a global batch."""

    def __init__(self, shape, global_batch, rank, world, direction=-1, precision=0, flags=0,
                 device=-1):
        from . import Plan
        self.start, self.count = shard_range(global_batch, rank, world)
        self.global_batch = global_batch
        self.plan = Plan(shape, self.count, direction, precision, flags, device)
