"""Continuous detectors (linear capsules, quadratic B-spline sweeps) against
the FP64 oracle: trajectory and segment flags outside the 1e-5 m band,
hit counts wherever no primitive pair is marginal."""
import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def sweep_setup(ctx, panda):
    sph = scenes.synth_spheres(panda, per_link=8, seed=0)
    mesh = scenes.sweep_scene()
    robot = rtcd.Robot(ctx, panda, spheres=sph)
    scene = rtcd.Scene.from_mesh(ctx, mesh)
    return robot, scene, O.Robot(panda, spheres=sph), O.Scene(mesh)


def _cmp(out, ref):
    tb = ref['traj_band'].astype(bool)
    m = (out['flags'] != ref['traj_hit']) & ~tb
    assert m.sum() == 0, 'trajectory flag mismatches at %s' % np.nonzero(m)[0][:20]
    if 'seg_flags' in out:
        sb = ref['seg_band'].astype(bool)
        ms = (out['seg_flags'] != ref['seg_hit']) & ~sb
        assert ms.sum() == 0, 'segment flag mismatches at %s' % np.nonzero(ms)[0][:20]
        # a trajectory is hit iff one of its segments is
        off = out['seg_off']
        for t in range(len(out['flags'])):
            assert out['flags'][t] == out['seg_flags'][off[t]:off[t + 1]].max(initial=0)
    if 'counts' in out:
        safe = ~ref['traj_marg'].astype(bool)
        mc = (out['counts'] != ref['traj_count']) & safe
        assert mc.sum() == 0, 'count mismatches at %s' % np.nonzero(mc)[0][:20]


def test_linear_parity(sweep_setup, panda):
    robot, scene, orob, osc = sweep_setup
    q, off = scenes.random_walk_trajectories(panda, 256, 32, seed=0)
    ref = O.sweep(False, orob, osc, q, off)
    det = rtcd.Detector(robot.ctx, 'Linear', robot, scene)
    _cmp(det.check(q, off, segments=True), ref)
    _cmp(det.check(q, off, counts=True, segments=True), ref)
    plain = det.check(q, off)
    _cmp(plain, ref)
    assert 0.05 < ref['traj_hit'].mean() < 0.99


def test_quadratic_parity_uneven(sweep_setup, panda):
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(192, 8, 64, seed=1)
    q, off = scenes.random_walk_trajectories(panda, 192, n_wp, seed=1)
    ref = O.sweep(True, orob, osc, q, off)
    det = rtcd.Detector(robot.ctx, 'Quadratic', robot, scene)
    _cmp(det.check(q, off, segments=True), ref)
    _cmp(det.check(q, off, counts=True), ref)
    ref_ne = O.sweep(True, orob, osc, q, off, endpoints=False)
    _cmp(det.check(q, off, segments=True, flags=rtcd.CHECK_NO_ENDPOINTS), ref_ne)


def test_quadratic_fit_weights_on_device_match_tables(sweep_setup, panda):
    """The device fit uses W = pinv(B): a trajectory whose waypoints lie on a
    quadratic B-spline is reproduced, so its sweep equals the spline's sweep."""
    robot, scene, orob, osc = sweep_setup
    q, off = scenes.random_walk_trajectories(panda, 64, 32, seed=5)
    det = rtcd.Detector(robot.ctx, 'Quadratic', robot, scene)
    ref = O.sweep(True, orob, osc, q, off)
    _cmp(det.check(q, off, segments=True), ref)


def test_short_and_single_trajectories(sweep_setup, panda):
    robot, scene, orob, osc = sweep_setup
    for kind, quad, wp in (('Linear', False, [2, 3, 2]), ('Quadratic', True, [3, 4, 5])):
        q, off = scenes.random_walk_trajectories(panda, 3, wp, seed=2)
        det = rtcd.Detector(robot.ctx, kind, robot, scene)
        _cmp(det.check(q, off, segments=True, counts=True), O.sweep(quad, orob, osc, q, off))
        one = det.check(q[:off[1]], off[:2])
        assert one['flags'][0] == det.check(q, off)['flags'][0]


def test_sweep_results_independent_of_batch(sweep_setup, panda):
    robot, scene, _, _ = sweep_setup
    n_wp = scenes.log_uniform_counts(64, 8, 40, seed=3)
    q, off = scenes.random_walk_trajectories(panda, 64, n_wp, seed=3)
    det = rtcd.Detector(robot.ctx, 'Quadratic', robot, scene)
    full = det.check(q, off)['flags']
    for a, b in ((0, 10), (10, 11), (11, 64)):
        sub_off = off[a:b + 1] - off[a]
        part = det.check(q[off[a]:off[b]], sub_off)['flags']
        assert np.array_equal(part, full[a:b])


def test_sweep_rejects_bad_offsets(sweep_setup):
    robot, scene, _, _ = sweep_setup
    det = rtcd.Detector(robot.ctx, 'Linear', robot, scene)
    with pytest.raises(rtcd.RTCDError):
        det.check(np.zeros((4, 7), np.float32), np.array([0, 3, 1], np.uint32))
    with pytest.raises(rtcd.RTCDError):
        det.check(np.zeros((4, 7), np.float32), np.array([0, 1], np.uint32))  # one waypoint
    qd = rtcd.Detector(robot.ctx, 'Quadratic', robot, scene)
    with pytest.raises(rtcd.RTCDError):
        qd.check(np.zeros((2, 7), np.float32), np.array([0, 2], np.uint32))


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_sweep_graph_replay_matches_direct_path(sweep_setup, panda, kind):
    """RTCD_CHECK_GRAPH for the sweeps: the first call captures, later calls
    with the same buffers and trajectory offsets replay; new waypoint contents
    give the same trajectory and segment flags as the direct path, and new
    offsets capture again."""
    import torch
    robot, scene, _, _ = sweep_setup
    det = rtcd.Detector(robot.ctx, kind, robot, scene)
    ref_det = rtcd.Detector(robot.ctx, kind, robot, scene)  # a direct call on `det` would retire its graph
    s = torch.cuda.Stream()
    for off_seed in (1, 2):
        counts = scenes.log_uniform_counts(40, 8, 40, seed=off_seed)
        off = np.zeros(41, np.uint32)
        off[1:] = np.cumsum(counts)
        nseg = int(rtcd.segment_offsets(det.kind, off)[-1])
        with torch.cuda.stream(s):
            qd = torch.zeros((int(off[-1]), 7), dtype=torch.float32, device='cuda')
            fd = torch.zeros(40, dtype=torch.uint8, device='cuda')
            sd = torch.zeros(nseg, dtype=torch.uint8, device='cuda')
            for seed in (31, 32, 33):
                q, _ = scenes.random_walk_trajectories(panda, 40, counts, seed=seed)
                qd.copy_(torch.from_numpy(q))
                det.check_device(qd, 40, fd, traj_off=off, seg_dev=sd, flags=rtcd.CHECK_GRAPH, stream=s.cuda_stream)
                det.sync(s.cuda_stream)
                ref = ref_det.check(q, off, segments=True)
                assert np.array_equal(fd.cpu().numpy(), ref['flags']), (off_seed, seed)
                assert np.array_equal(sd.cpu().numpy(), ref['seg_flags']), (off_seed, seed)


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_binary_and_wide_trees_agree(sweep_setup, panda, kind):
    """The lane and warp descents over the binary edge tree (stage_b_form 1)
    and over its 4-wide copy (the default) give the oracle's flags and counts,
    with short light budgets so the heavy pass takes many units."""
    robot, scene, orob, osc = sweep_setup
    n_wp = 24 if kind == 'Linear' else scenes.log_uniform_counts(128, 8, 48, seed=3)
    q, off = scenes.random_walk_trajectories(panda, 128, n_wp, seed=3)
    ref = O.sweep(kind == 'Quadratic', orob, osc, q, off)
    for form in (0, 1):
        for light in (4, 0):
            det = rtcd.Detector(robot.ctx, kind, robot, scene, stage_b_form=form, light_steps=light)
            _cmp(det.check(q, off, segments=True), ref)
            _cmp(det.check(q, off, counts=True, segments=True), ref)
            det.close()


def test_graph_with_host_buffers(sweep_setup, panda):
    """RTCD_CHECK_GRAPH with host arrays on a sweep detector: replays with new
    waypoints under the same trajectory offsets equal the plain host path
    (trajectory flags, segment flags, counts)."""
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(96, 8, 40, seed=4)
    runs = [scenes.random_walk_trajectories(panda, 96, n_wp, seed=s) for s in (4, 5)]
    off = runs[0][1]
    assert all(np.array_equal(o, off) for _, o in runs)
    for kind in ('Linear', 'Quadratic'):
        det = rtcd.Detector(robot.ctx, kind, robot, scene)
        refs = [det.check(q, off, counts=True, segments=True) for q, _ in runs]
        for (q, _), ref in zip(runs + runs, refs + refs):
            got = det.check(q, off, counts=True, segments=True, flags=rtcd.CHECK_GRAPH)
            for k in ('flags', 'seg_flags', 'counts'):
                assert np.array_equal(got[k], ref[k]), k
        det.close()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_staged_and_unstaged_light_pass_agree(sweep_setup, panda, kind):
    """The staged light pass (each trajectory's FK and fit in shared memory)
    and the unstaged one (centres and control points through global memory)
    give the same trajectory and segment flags, and equal counts wherever the
    oracle sees no marginal pair; a batch with a trajectory too long for the
    staging falls back to the unstaged pass with the same results."""
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(1200, 8, 64, seed=11)
    n_wp[1100] = 700  # longer than the staging holds: the whole batch takes the unstaged pass
    q, off = scenes.random_walk_trajectories(panda, 1200, n_wp, seed=11)
    # one block per SM: 1,100 trajectories are enough for the staged pass (at least 4 per block)
    staged = rtcd.Detector(robot.ctx, kind, robot, scene, traverse_blocks_per_sm=1)
    unstaged = rtcd.Detector(robot.ctx, kind, robot, scene, sweep_unstaged=1)
    quad = kind == 'Quadratic'
    for surface in (False, True):
        for a, b, path in ((q[:off[1100]], off[:1101], 1), (q, off, 0)):
            staged.check(a, b, surface=surface)
            assert staged.stats()['path_flags'] & 1 == path
            ref = O.sweep(quad, orob, osc, a, b, surface=surface)
            x = staged.check(a, b, segments=True, counts=True, surface=surface)
            y = unstaged.check(a, b, segments=True, counts=True, surface=surface)
            _cmp(x, ref)
            _cmp(y, ref)
            # the two passes round the sphere centres differently (the fit on transforms or on
            # centres): they may differ only on segments the oracle puts in the band
            diff = x['seg_flags'] != y['seg_flags']
            assert not (diff & (ref['seg_band'] == 0)).any()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_grouped_staging_matches_one_at_a_time(sweep_setup, panda, kind):
    """The staged light pass working through groups of trajectories (2, 3 or
    8 staged together, the batch not a multiple of the group) gives exactly
    the flags, segment flags and counts of one trajectory at a time: each
    trajectory's FK and fit run the same arithmetic in its own slot."""
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(1201, 3, 64, seed=12)
    q, off = scenes.random_walk_trajectories(panda, 1201, n_wp, seed=12)
    one = rtcd.Detector(robot.ctx, kind, robot, scene, traverse_blocks_per_sm=1, sweep_group=1)
    for surface in (False, True):
        x = one.check(q, off, segments=True, counts=True, surface=surface)
        assert one.stats()['path_flags'] & 1 == 1
        xf = one.check(q, off, segments=True, surface=surface)
        for group in (2, 3, 8):
            det = rtcd.Detector(robot.ctx, kind, robot, scene, traverse_blocks_per_sm=1, sweep_group=group)
            y = det.check(q, off, segments=True, counts=True, surface=surface)
            assert det.stats()['path_flags'] & 1 == 1
            for k in ('flags', 'seg_flags', 'counts'):
                assert np.array_equal(x[k], y[k]), (group, k)
            yf = det.check(q, off, segments=True, surface=surface)
            for k in ('flags', 'seg_flags'):
                assert np.array_equal(xf[k], yf[k]), (group, k)
            det.close()
    ref = O.sweep(kind == 'Quadratic', orob, osc, q[:off[64]], off[:65])
    got = one.check(q[:off[64]], off[:65], segments=True, counts=True)
    _cmp(got, ref)
    one.close()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_heavy_split_pass_keeps_results(sweep_setup, panda, kind):
    """Heavy-pass units that hand their open frontier to the split pass after
    1, 4 or the default 32 frontier steps, or never: the same flags, segment
    flags and counts (every node is expanded exactly once), in both
    semantics."""
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(600, 3, 64, seed=13)
    q, off = scenes.random_walk_trajectories(panda, 600, n_wp, seed=13)
    never = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=4, sweep_heavy_steps=0xFFFFFFFF)
    for surface in (False, True):
        x = never.check(q, off, segments=True, counts=True, surface=surface)
        assert never.stats()['deferred'] > 0
        xf = never.check(q, off, segments=True, surface=surface)
        for steps in (1, 4, 0):
            det = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=4, sweep_heavy_steps=steps)
            y = det.check(q, off, segments=True, counts=True, surface=surface)
            for k in ('flags', 'seg_flags', 'counts'):
                assert np.array_equal(x[k], y[k]), (steps, k)
            yf = det.check(q, off, segments=True, surface=surface)
            for k in ('flags', 'seg_flags'):
                assert np.array_equal(xf[k], yf[k]), (steps, k)
            det.close()
    ref = O.sweep(kind == 'Quadratic', orob, osc, q[:off[100]], off[:101])
    det = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=4, sweep_heavy_steps=1)
    _cmp(det.check(q[:off[100]], off[:101], segments=True, counts=True), ref)
    det.close()
    never.close()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_split_list_overflow_keeps_results(sweep_setup, panda, kind):
    """A batch whose split list (one slot per unit the light pass can defer)
    cannot hold every frontier handed to it: 64 trajectories parked at the
    pose that collides most (every waypoint the same), counted (no early
    exit), a light budget of one visit and heavy units splitting after one
    step.  A reservation that does not fit stays with its warp and its slots
    below the capacity are blanked, so the flags, segment flags and counts
    equal the never-splitting run's, on fresh and on reused device memory
    (repeated detectors)."""
    robot, scene, orob, osc = sweep_setup
    cand = scenes.uniform_poses(panda, 512, seed=22)
    probe = rtcd.Detector(robot.ctx, 'Linear', robot, scene)
    pairs = np.repeat(cand, 2, axis=0)
    hits = probe.check(pairs, np.arange(0, 2 * len(cand) + 1, 2, dtype=np.uint32), counts=True)['counts']
    probe.close()
    pose = cand[int(np.argmax(hits))]
    q = np.tile(pose, (64 * 16, 1)).astype(np.float32)
    off = np.arange(0, 64 * 16 + 1, 16, dtype=np.uint32)
    never = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=1, sweep_heavy_steps=0xFFFFFFFF)
    x = never.check(q, off, segments=True, counts=True)
    assert x['flags'].all() and never.stats()['deferred'] > 10000
    for _ in range(3):
        det = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=1, sweep_heavy_steps=1)
        y = det.check(q, off, segments=True, counts=True)
        for k in ('flags', 'seg_flags', 'counts'):
            assert np.array_equal(x[k], y[k]), k
        det.close()
    never.close()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_page_locked_waypoints_match_pageable(sweep_setup, panda, kind):
    """Sweep host calls with waypoints in page-locked memory (direct DMA, in
    the direct path and in the graph) give the pageable calls' trajectory and
    segment flags; a pinned array rewritten in place is read afresh."""
    import torch
    robot, scene, _, _ = sweep_setup
    n_wp = scenes.log_uniform_counts(160, 8, 48, seed=7)
    walks = [scenes.random_walk_trajectories(panda, 160, n_wp, seed=s) for s in (7, 8)]
    off = walks[0][1]
    assert all(np.array_equal(w[1], off) for w in walks)
    det = rtcd.Detector(robot.ctx, kind, robot, scene)
    refs = [det.check(q, off, segments=True) for q, _ in walks]
    assert any(r['flags'].any() for r in refs)
    pin = torch.empty(walks[0][0].shape, dtype=torch.float32).pin_memory().numpy()
    for graph in (0, rtcd.CHECK_GRAPH):
        for i in (0, 1, 0):
            pin[...] = walks[i][0]
            got = det.check(pin, off, segments=True, flags=graph)
            assert np.array_equal(got['flags'], refs[i]['flags'])
            assert np.array_equal(got['seg_flags'], refs[i]['seg_flags'])
            got = det.check(walks[1 - i][0], off, flags=graph)
            assert np.array_equal(got['flags'], refs[1 - i]['flags'])
    det.close()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_descend_cap_keeps_results(sweep_setup, panda, kind):
    """The light pass's per-descent visit cap only changes when idle lanes
    take new units: trajectory flags, segment flags and counts are the same
    at caps 1, 3 (the default), 4 and none, with and without the heavy pass."""
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(200, 8, 40, seed=11)
    q, off = scenes.random_walk_trajectories(panda, 200, n_wp, seed=11)
    ref = O.sweep(kind == 'Quadratic', orob, osc, q, off)
    outs = []
    for light in (0, 0xFFFFFFFF):
        for cap in (1, 0, 4, 0xFFFFFFFF):
            det = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=light, sweep_descend_cap=cap)
            seg = det.check(q, off, segments=True)
            cnt = det.check(q, off, counts=True)
            _cmp(seg, ref)
            _cmp(cnt, ref)
            outs.append((seg['flags'], seg['seg_flags'], cnt['counts']))
            det.close()
    for o in outs[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(o, outs[0]))


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
@pytest.mark.parametrize('surface', [False, True])
def test_wide_heavy_pass_keeps_results(sweep_setup, panda, kind, surface):
    """The heavy and split passes on the 4-wide edge tree (four lanes per
    node) give the binary tree's trajectory flags, segment flags and counts,
    with a light budget small enough to send most units there and the split
    pass forced on; the solid semantics also match the oracle."""
    robot, scene, orob, osc = sweep_setup
    n_wp = scenes.log_uniform_counts(160, 8, 40, seed=13)
    q, off = scenes.random_walk_trajectories(panda, 160, n_wp, seed=13)
    outs = []
    for wide in (0, 1):
        for heavy_steps in (1, 0xFFFFFFFF):
            det = rtcd.Detector(robot.ctx, kind, robot, scene, light_steps=2, sweep_heavy_steps=heavy_steps,
                                sweep_heavy_wide=wide)
            seg = det.check(q, off, segments=True, surface=surface)
            cnt = det.check(q, off, counts=True, surface=surface)
            assert det.stats()['deferred'] > 0
            outs.append((seg['flags'], seg['seg_flags'], cnt['counts']))
            det.close()
    for o in outs[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(o, outs[0]))
    if not surface:
        ref = O.sweep(kind == 'Quadratic', orob, osc, q, off)
        _cmp({'flags': outs[0][0], 'counts': outs[0][2]}, ref)
