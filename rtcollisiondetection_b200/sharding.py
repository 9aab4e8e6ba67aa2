"""Multi-GPU sharding of a query batch: one process per GPU.

Poses and trajectories are independent, so a batch splits into contiguous
ranges, one per rank, with no exchange on the data path; each rank keeps its
own resident copy of the scene and robot (built from the same inputs, so the
trees are identical).  Trajectory ranges are balanced by waypoint count.  The
only exchange is the concatenation of the uint8 result flags, done with
``all_gather`` on the process group (NCCL over NVLink on GPUs, gloo on CPU).
"""
import numpy as np


def shard_bounds(n, world, weights=None):
    """Contiguous [start, stop) per rank.  ``weights`` (per unit, e.g. the
    waypoint count of each trajectory) balances the cumulative weight;
    without it the split is by count."""
    if world < 1:
        raise ValueError('world must be >= 1')
    if weights is None:
        base, extra = divmod(n, world)
        sizes = [base + (1 if r < extra else 0) for r in range(world)]
        bounds = np.concatenate([[0], np.cumsum(sizes)])
    else:
        w = np.asarray(weights, np.float64)
        if len(w) != n:
            raise ValueError('one weight per unit')
        c = np.concatenate([[0.0], np.cumsum(w)])
        targets = c[-1] * np.arange(world + 1) / world
        bounds = np.searchsorted(c, targets, side='left')
        bounds[0], bounds[-1] = 0, n
        bounds = np.maximum.accumulate(bounds)
    return [(int(bounds[r]), int(bounds[r + 1])) for r in range(world)]


def shard_trajectories(traj_off, world, rank):
    """This rank's trajectory range of a batch: (t0, t1, waypoint rows r0:r1,
    local offsets)."""
    traj_off = np.asarray(traj_off, np.int64)
    n = len(traj_off) - 1
    t0, t1 = shard_bounds(n, world, np.diff(traj_off))[rank]
    r0, r1 = int(traj_off[t0]), int(traj_off[t1])
    return t0, t1, r0, r1, (traj_off[t0:t1 + 1] - r0).astype(np.uint32)


def gather_flags(local, n_total, world, group=None, device=None):
    """All-gather every rank's flags into one uint8 array of length n_total
    (ranks hold contiguous, count-balanced ranges).  Uses torch.distributed."""
    import torch
    import torch.distributed as dist
    bounds = shard_bounds(n_total, world) if world > 1 else [(0, n_total)]
    width = max(b - a for a, b in bounds)
    dev = device if device is not None else 'cpu'
    t = torch.zeros(width, dtype=torch.uint8, device=dev)
    src = torch.as_tensor(np.asarray(local, np.uint8), device=dev)
    t[:len(src)] = src
    if world == 1:
        return t[:n_total].cpu().numpy()
    parts = [torch.zeros(width, dtype=torch.uint8, device=dev) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return np.concatenate([parts[r][:b - a].cpu().numpy() for r, (a, b) in enumerate(bounds)])


def max_over_ranks(value, group=None, device=None):
    """The largest value over ranks (step times are reported as the max)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device if device is not None else 'cpu')
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
