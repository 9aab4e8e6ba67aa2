"""Pose/trajectory sharding across ranks: host logic and a world_size-2 gloo
run on CPU (the device detectors are replaced by the oracle here: the test
covers the split and the flag exchange, not the kernels)."""
import os
import socket

import numpy as np
import pytest

from rtcollisiondetection_b200 import sharding


def test_count_split_is_contiguous_and_balanced():
    for n in (0, 1, 7, 65536, 65537):
        for w in (1, 2, 3, 8):
            b = sharding.shard_bounds(n, w)
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
            sizes = [y - x for x, y in b]
            assert max(sizes) - min(sizes) <= 1


def test_weighted_split_balances_waypoints():
    rng = np.random.default_rng(0)
    w = rng.integers(8, 129, size=1000)
    b = sharding.shard_bounds(1000, 4, w)
    loads = [w[x:y].sum() for x, y in b]
    assert max(loads) - min(loads) <= 2 * w.max()
    off = np.concatenate([[0], np.cumsum(w)])
    t0, t1, r0, r1, loc = sharding.shard_trajectories(off, 4, 2)
    assert (t0, t1) == b[2] and r0 == off[t0] and r1 == off[t1] and loc[-1] == r1 - r0


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, out):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from rtcollisiondetection_b200 import scenes
        model = scenes.load_panda()
        mesh = scenes.discrete_small()
        a, b = sharding.shard_bounds(len(q), world)[rank]
        local = O.discrete(O.ROBOT_TO_OBS, O.Robot(model), O.Scene(mesh), q[a:b])['hit']
        flags = sharding.gather_flags(local, len(q), world)
        t = sharding.max_over_ranks(float(rank + 1))
        if rank == 0:
            out.put((flags, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_check_matches_single_rank():
    import torch.multiprocessing as mp
    from oracle import oracle as O
    from rtcollisiondetection_b200 import scenes
    model = scenes.load_panda()
    q = scenes.uniform_poses(model, 101, seed=4)
    whole = O.discrete(O.ROBOT_TO_OBS, O.Robot(model), O.Scene(scenes.discrete_small()), q)['hit']
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, out)) for r in range(2)]
    for p in procs:
        p.start()
    flags, tmax = out.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.array_equal(flags, whole)
    assert tmax == 2.0
