"""The continuous-batching server: requests of mixed kinds, sizes and scenes
submitted concurrently from several threads; every result must equal the
result of the same request checked alone (flags, segment flags, counts)."""
import threading

import numpy as np
import pytest

from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def world(ctx, panda):
    sph = scenes.synth_spheres(panda)
    robot = rtcd.Robot(ctx, panda, spheres=sph)
    small = rtcd.Scene.from_mesh(ctx, scenes.discrete_small())
    sweep = rtcd.Scene.from_mesh(ctx, scenes.sweep_scene())
    dets = {
        'r2o_small': rtcd.Detector(ctx, 'RobotToObs', robot, small),
        'o2r_small': rtcd.Detector(ctx, 'ObsToRobot', robot, small),
        'r2o_sweep': rtcd.Detector(ctx, 'RobotToObs', robot, sweep),
        'lin': rtcd.Detector(ctx, 'Linear', robot, sweep),
        'quad': rtcd.Detector(ctx, 'Quadratic', robot, sweep),
    }
    return robot, dets


def _requests(panda, n_req, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n_req):
        kind = ['r2o_small', 'o2r_small', 'r2o_sweep', 'lin', 'quad'][i % 5]
        counts = bool(rng.integers(0, 2))
        if kind in ('lin', 'quad'):
            nt = int(np.exp(rng.uniform(0, np.log(48))))
            wp = scenes.log_uniform_counts(nt, 8, 40, seed=seed * 1000 + i)
            q, off = scenes.random_walk_trajectories(panda, nt, wp, seed=seed * 1000 + i)
        else:
            n = int(np.exp(rng.uniform(0, np.log(700))))
            q, off = scenes.uniform_poses(panda, n, seed=seed * 1000 + i), None
        reqs.append((kind, q, off, counts))
    return reqs


def test_server_results_equal_alone(world, panda):
    _, dets = world
    server = rtcd.Server(dets['lin'].ctx, slots=3, max_batch_units=4096)
    reqs = _requests(panda, 60, seed=3)
    tickets = [None] * len(reqs)

    def submitter(idx):
        for i in idx:
            kind, q, off, counts = reqs[i]
            tickets[i] = server.submit(dets[kind], q, off, counts=counts)

    threads = [threading.Thread(target=submitter, args=(range(k, len(reqs), 3),)) for k in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    results = [server.wait(t, timeout_ms=120000) for t in tickets]
    st = server.stats()
    server.close()
    assert st['completed'] == len(reqs) and st['failed'] == 0
    assert st['batches'] <= len(reqs)
    assert st['p99_ms'] >= st['p50_ms'] > 0
    for (kind, q, off, counts), got in zip(reqs, results):
        det = dets[kind]
        alone = det.check(q, off, counts=counts, segments=det.sweep)
        assert np.array_equal(got['flags'], alone['flags']), kind
        if counts:
            assert np.array_equal(got['counts'], alone['counts']), kind
        if det.sweep:
            assert np.array_equal(got['seg_flags'], alone['seg_flags']), kind


def test_server_merges_queued_requests(world, panda):
    _, dets = world
    server = rtcd.Server(dets['r2o_small'].ctx, slots=1, max_batch_units=65536)
    qs = [scenes.uniform_poses(panda, 50, seed=100 + i) for i in range(40)]
    tickets = [server.submit(dets['r2o_small'], q) for q in qs]
    outs = [server.wait(t) for t in tickets]
    st = server.stats()
    server.close()
    assert st['batches'] < len(qs)           # queued requests shared launches
    whole = dets['r2o_small'].check(np.concatenate(qs))['flags']
    assert np.array_equal(np.concatenate([o['flags'] for o in outs]), whole)


def test_server_fast_lane_prepared(world, panda):
    """A prepared server with one fast slot (requests of <= 256 units on a
    high-priority stream) and two bulk slots at 25 % residency: small and
    large requests interleaved, results equal to the requests checked alone."""
    _, dets = world
    server = rtcd.Server(dets['lin'].ctx, slots=3, max_batch_units=8192, fast_slots=1, fast_max_units=256,
                         bulk_share=25)
    for k in ('r2o_small', 'o2r_small', 'lin', 'quad'):
        server.prepare(dets[k], 4096)
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(40):
        k = ['r2o_small', 'o2r_small', 'lin', 'quad'][i % 4]
        big = i % 3 == 0
        if k in ('lin', 'quad'):
            nt = 200 if big else int(rng.integers(1, 12))
            q, off = scenes.random_walk_trajectories(panda, nt, scenes.log_uniform_counts(nt, 8, 24, seed=i), seed=i)
        else:
            q, off = scenes.uniform_poses(panda, 3000 if big else int(rng.integers(1, 200)), seed=500 + i), None
        reqs.append((k, q, off))
    tickets = [server.submit(dets[k], q, off) for k, q, off in reqs]
    outs = [server.wait(t, timeout_ms=120000) for t in tickets]
    st = server.stats()
    server.close()
    assert st['completed'] == len(reqs) and st['failed'] == 0
    for (k, q, off), got in zip(reqs, outs):
        alone = dets[k].check(q, off, segments=dets[k].sweep)
        assert np.array_equal(got['flags'], alone['flags']), k
        if dets[k].sweep:
            assert np.array_equal(got['seg_flags'], alone['seg_flags']), k


def test_prepared_server_serves_without_reallocation(world, panda):
    """After rtcd_server_prepare, requests of any shape within the prepared
    size - discrete batches, sweeps of 1 to 60 trajectories of 2/3 to 128
    waypoints (staged and unstaged light passes), flags-only and counting,
    solid and reference semantics - run without a workspace re-allocation
    (each would synchronise the device and stall every slot), and their
    results equal the requests checked alone."""
    _, dets = world
    server = rtcd.Server(dets['lin'].ctx, slots=3, max_batch_units=8192, fast_slots=1, fast_max_units=256)
    for k in ('r2o_small', 'o2r_small', 'lin', 'quad'):
        server.prepare(dets[k], 8192)
    server.reset_stats()
    rng = np.random.default_rng(21)
    reqs = []
    for i in range(48):
        k = ['r2o_small', 'o2r_small', 'lin', 'quad'][i % 4]
        counts = bool(rng.integers(0, 2))
        surface = bool(rng.integers(0, 2))
        if k in ('lin', 'quad'):
            nt = int(rng.integers(1, 61))
            lo = 2 if k == 'lin' else 3
            wp = np.minimum(scenes.log_uniform_counts(nt, lo, 128, seed=700 + i), 8192 // nt)
            q, off = scenes.random_walk_trajectories(panda, nt, np.maximum(wp, lo), seed=700 + i)
        else:
            q, off, surface = scenes.uniform_poses(panda, int(rng.integers(1, 4097)), seed=900 + i), None, False
        reqs.append((k, q, off, counts, surface))
    tickets = [server.submit(dets[k], q, off, counts=c, surface=sf) for k, q, off, c, sf in reqs]
    outs = [server.wait(t, timeout_ms=120000) for t in tickets]
    st = server.stats()
    server.close()
    assert st['completed'] == len(reqs) and st['failed'] == 0
    assert st['workspace_grows'] == 0, st
    for (k, q, off, c, sf), got in zip(reqs, outs):
        alone = dets[k].check(q, off, segments=dets[k].sweep, counts=c, surface=sf)
        assert np.array_equal(got['flags'], alone['flags']), k
        if c:
            assert np.array_equal(got['counts'], alone['counts']), k
        if dets[k].sweep:
            assert np.array_equal(got['seg_flags'], alone['seg_flags']), k


def test_server_rejects_bad_config(world):
    _, dets = world
    with pytest.raises(rtcd.RTCDError):
        rtcd.Server(dets['lin'].ctx, slots=2, fast_slots=2)        # no slot would take large requests
    with pytest.raises(rtcd.RTCDError):
        rtcd.Server(dets['lin'].ctx, slots=2, bulk_share=150)


def test_server_rejects_bad_requests(world, panda):
    _, dets = world
    server = rtcd.Server(dets['lin'].ctx, slots=1)
    with pytest.raises(rtcd.RTCDError):
        server.submit(dets['lin'], np.zeros((4, 7), np.float32), np.array([0, 3, 1], np.uint32))
    with pytest.raises(rtcd.RTCDError):
        rtcd._ok(rtcd.lib().rtcd_server_wait(server.h, rtcd.C.c_uint64(12345), rtcd.C.c_int32(0), None, None, None,
                                             None))
    server.close()


def test_memory_admission_serialises_launches(world, panda):
    """Admission by memory: with a budget no larger than one launch, launches
    run one at a time (the peak of the bytes in flight is one launch's), with
    a budget of several launches more run at once; every result still equals
    the request checked alone."""
    _, dets = world
    det = dets['r2o_small']
    qs = [scenes.uniform_poses(panda, 512, seed=100 + i) for i in range(24)]
    alone = [det.check(q)['flags'] for q in qs]

    def serve(budget):
        # one request per launch (max_batch_units = the request size) on two bulk slots that could
        # overlap (the fast slot takes only requests of at most 256 poses: none here)
        srv = rtcd.Server(det.ctx, slots=3, fast_slots=1, fast_max_units=256, max_batch_units=512,
                          memory_budget=budget)
        srv.prepare(det, 512)
        srv.reset_stats()
        ts = [srv.submit(det, q) for q in qs]
        outs = [srv.wait(t)['flags'] for t in ts]
        st = srv.stats()
        srv.close()
        for a, b in zip(outs, alone):
            assert np.array_equal(a, b)
        assert st['completed'] == len(qs) and st['batches'] == len(qs)
        return st['inflight_bytes_peak']

    one = serve(1)                      # smaller than any launch: each is admitted only when none is in flight
    assert one > 0
    assert serve(one) == one            # exactly one launch's bytes: still one at a time
    assert serve(2 * one) <= 2 * one    # two launches at most
    assert one <= serve(1 << 40) <= 2 * one  # unbounded: as many as the two bulk slots allow
