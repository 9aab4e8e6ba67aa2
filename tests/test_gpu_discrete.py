"""Discrete detectors (ObsToRobot, RobotToObs) against the FP64 oracle.

Flags must agree on every pose outside the 1e-5 m band; the upstream hit
counts must agree on every pose with no marginal primitive pair."""
import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu
KINDS = [('ObsToRobot', O.OBS_TO_ROBOT), ('RobotToObs', O.ROBOT_TO_OBS)]


@pytest.fixture(scope='module')
def setup(ctx, panda, small_scene):
    robot = rtcd.Robot(ctx, panda)
    scene = rtcd.Scene.from_mesh(ctx, small_scene)
    orc = (O.Robot(panda), O.Scene(small_scene))
    return robot, scene, orc


def _compare(out, ref, counts=True):
    band = ref['band'].astype(bool)
    mism = (out['flags'] != ref['hit']) & ~band
    assert mism.sum() == 0, 'flag mismatches outside the band at poses %s' % np.nonzero(mism)[0][:20]
    if counts:
        safe = ~ref['marg'].astype(bool)
        cm = (out['counts'] != ref['count']) & safe
        assert cm.sum() == 0, 'count mismatches at %s' % np.nonzero(cm)[0][:20]
        assert np.array_equal(out['counts'] > 0, out['flags'] > 0)


@pytest.mark.parametrize('name,okind', KINDS)
def test_small_scene_parity(setup, panda, name, okind):
    robot, scene, (orob, oscene) = setup
    q = scenes.uniform_poses(panda, 1024, seed=0)
    ref = O.discrete(okind, orob, oscene, q)
    det = rtcd.Detector(robot.ctx, name, robot, scene)
    flags_only = det.check(q)
    with_counts = det.check(q, counts=True)
    _compare(with_counts, ref)
    assert np.array_equal(flags_only['flags'], with_counts['flags'])
    assert 0.2 < ref['hit'].mean() < 0.9  # the workload is not trivial


@pytest.mark.parametrize('name,okind', KINDS)
def test_cull_plain_and_device_paths_agree(setup, panda, name, okind):
    import torch
    robot, scene, _ = setup
    q = scenes.uniform_poses(panda, 777, seed=11)
    det = rtcd.Detector(robot.ctx, name, robot, scene, frame_size=64)
    a = det.check(q, counts=True)
    b = det.check(q, counts=True, flags=rtcd.CHECK_NO_CULL)
    c = det.check(q, counts=True, flags=rtcd.CHECK_PLAIN)
    assert np.array_equal(a['flags'], b['flags']) and np.array_equal(a['counts'], b['counts'])
    assert np.array_equal(a['flags'], c['flags']) and np.array_equal(a['counts'], c['counts'])
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        qd = torch.from_numpy(q).cuda()
        fd = torch.zeros(len(q), dtype=torch.uint8, device='cuda')
        cd = torch.zeros(len(q), dtype=torch.int32, device='cuda')
        det.check_device(qd, len(q), fd, counts_dev=cd, stream=s.cuda_stream)
        det.sync(s.cuda_stream)
    assert np.array_equal(fd.cpu().numpy(), a['flags'])
    assert np.array_equal(cd.cpu().numpy().astype(np.uint32), a['counts'])


@pytest.mark.parametrize('name,okind', KINDS)
@pytest.mark.parametrize('light', [1, 0, 0xFFFFFFFF])
def test_stage_b_forms_agree(setup, panda, name, okind, light):
    """Packet and per-lane stage B at two chunk lengths each and the fused
    stage A+B, with every
    candidate spilled to the heavy pass (budget 1), the default budget, and
    no heavy pass: identical flags and counts, and the flags agree with the
    oracle outside the band."""
    robot, scene, (orob, oscene) = setup
    q = scenes.uniform_poses(panda, 600, seed=21)
    dets = [rtcd.Detector(robot.ctx, name, robot, scene, light_steps=light, stage_b_form=f, stage_b_chunk=k)
            for f, k in ((1, 1), (1, 64), (2, 1), (2, 4), (3, 0), (3, 1), (4, 0), (4, 1))]
    flags_only = [d.check(q) for d in dets]
    counted = [d.check(q, counts=True) for d in dets]
    for o in flags_only + counted:
        assert np.array_equal(o['flags'], counted[0]['flags'])
    for o in counted[1:]:
        assert np.array_equal(o['counts'], counted[0]['counts'])
    ref = O.discrete(okind, orob, oscene, q)
    _compare(counted[0], ref)


@pytest.mark.parametrize('name,okind', KINDS)
def test_edge_cases(setup, panda, name, okind):
    robot, scene, (orob, oscene) = setup
    det = rtcd.Detector(robot.ctx, name, robot, scene)
    # single pose, the joint limits, repeated poses
    q = np.stack([panda['lower'], panda['upper'], 0.5 * (panda['lower'] + panda['upper'])]).astype(np.float32)
    q = np.concatenate([q, q[:1].repeat(5, 0)])
    ref = O.discrete(okind, orob, oscene, q)
    _compare(det.check(q, counts=True), ref)
    one = det.check(q[:1])
    assert one['flags'][0] == det.check(q)['flags'][0]


def test_empty_scene_and_far_scene(ctx, panda):
    robot = rtcd.Robot(ctx, panda)
    far = scenes.random_scene(3, 3, 1, seed=5)
    far.verts[:] += np.float32(50.0)
    for mesh in (far,):
        sc = rtcd.Scene.from_mesh(ctx, mesh)
        for name in ('ObsToRobot', 'RobotToObs'):
            det = rtcd.Detector(ctx, name, robot, sc)
            out = det.check(scenes.uniform_poses(panda, 100), counts=True)
            assert out['flags'].sum() == 0 and out['counts'].sum() == 0


def test_single_triangle_scene(ctx, panda):
    """A single large triangle through the robot's reach; brute-force oracle."""
    robot = rtcd.Robot(ctx, panda)
    v = np.array([[-1, -1, 0.5], [2, -1, 0.5], [-1, 2, 0.5]], np.float32)
    t = np.array([[0, 1, 2]], np.uint32)
    mesh = scenes.Mesh(v, t, np.array([0, 1], np.uint32))
    sc = rtcd.Scene.from_mesh(ctx, mesh)
    q = scenes.uniform_poses(panda, 256, seed=9)
    orob, osc = O.Robot(panda), O.Scene(mesh)
    for name, okind in KINDS:
        det = rtcd.Detector(ctx, name, robot, sc)
        _compare(det.check(q, counts=True), O.discrete(okind, orob, osc, q))


def test_invalid_arguments(ctx, panda, small_scene):
    robot = rtcd.Robot(ctx, panda)
    with pytest.raises(rtcd.RTCDError):
        rtcd.Scene(ctx, small_scene.verts, np.array([[0, 1, 10 ** 7]], np.uint32))
    sc = rtcd.Scene.from_mesh(ctx, small_scene)
    with pytest.raises(rtcd.RTCDError):
        rtcd.Detector(ctx, 7, robot, sc)
    det = rtcd.Detector(ctx, 'RobotToObs', robot, sc)
    with pytest.raises(rtcd.RTCDError):
        det.check(np.zeros((4, 7), np.float32), segments=True, traj_off=np.array([0, 4], np.uint32))


@pytest.mark.parametrize('name', ['RobotToObs', 'ObsToRobot'])
def test_graph_replay_matches_direct_path(setup, panda, name):
    """RTCD_CHECK_GRAPH: the first call captures the launch sequence, later
    calls with the same buffers replay it; new pose contents in the same
    buffer give the same flags and counts as the direct path."""
    import torch
    robot, scene, _ = setup
    det = rtcd.Detector(robot.ctx, name, robot, scene)
    ref_det = rtcd.Detector(robot.ctx, name, robot, scene)  # a direct call on `det` would retire its graph
    s = torch.cuda.Stream()
    n = 600
    with torch.cuda.stream(s):
        qd = torch.zeros((n, 7), dtype=torch.float32, device='cuda')
        fd = torch.zeros(n, dtype=torch.uint8, device='cuda')
        cd = torch.zeros(n, dtype=torch.int32, device='cuda')
        for seed in (21, 22, 23):
            q = scenes.uniform_poses(panda, n, seed=seed)
            qd.copy_(torch.from_numpy(q))
            det.check_device(qd, n, fd, counts_dev=cd, flags=rtcd.CHECK_GRAPH, stream=s.cuda_stream)
            det.sync(s.cuda_stream)
            ref = ref_det.check(q, counts=True)
            assert np.array_equal(fd.cpu().numpy(), ref['flags']), seed
            assert np.array_equal(cd.cpu().numpy().astype(np.uint32), ref['counts']), seed


def _tiny_box_scene(n_boxes, seed, extent=0.012):
    """Small cubes scattered over the robot's reach, plus the small shelf scene."""
    rng = np.random.default_rng(seed)
    base = scenes.discrete_small()
    verts, tris, off = [base.verts], [base.tris], list(base.obstacle_tri_off)
    nv = len(base.verts)
    for _ in range(n_boxes):
        c = rng.uniform([-0.6, -0.6, 0.0], [0.6, 0.6, 1.0])
        v, t = scenes.box_mesh(c, [extent] * 3)
        verts.append(v.astype(np.float32))
        tris.append(t + nv)
        nv += len(v)
        off.append(off[-1] + len(t))
    return scenes.Mesh(np.concatenate(verts), np.concatenate(tris), off)


@pytest.mark.parametrize('name,okind', KINDS)
def test_containment_matches_oracle(ctx, panda, name, okind):
    """RTCD_CHECK_CONTAINMENT: flag 1 where a surface crossing exists, 2 where
    the oracle finds a link inside an obstacle or an obstacle inside a link
    (ray parity) and no crossing; compared outside both bands."""
    mesh = _tiny_box_scene(400, seed=7)
    robot = rtcd.Robot(ctx, panda)
    sc = rtcd.Scene.from_mesh(ctx, mesh)
    q = scenes.uniform_poses(panda, 512, seed=8)
    det = rtcd.Detector(ctx, name, robot, sc)
    out = det.check(q, flags=rtcd.CHECK_CONTAINMENT)['flags']
    plain = det.check(q)['flags']
    assert np.array_equal(out & 1, plain)                      # the surface flags are unchanged
    orob, osc = O.Robot(panda), O.Scene(mesh)
    ref = O.discrete(okind, orob, osc, q)
    cont = O.containment(orob, osc, q, skip=ref['hit'])
    ok = (ref['band'] == 0) & (cont['band'] == 0)
    assert np.array_equal(out[ok] & 1, ref['hit'][ok])
    assert np.array_equal((out[ok] >> 1) & 1, cont['contain'][ok])
    assert cont['contain'][ok].sum() >= 3                       # the case is exercised
    assert ok.mean() > 0.95


def test_containment_enclosing_box(ctx, panda):
    robot = rtcd.Robot(ctx, panda)
    v, t = scenes.box_mesh([0, 0, 0.5], [6, 6, 6])
    sc = rtcd.Scene.from_mesh(ctx, scenes.Mesh(v, t, [0, 12]))
    q = scenes.uniform_poses(panda, 64, seed=9)
    for name in ('ObsToRobot', 'RobotToObs'):
        det = rtcd.Detector(ctx, name, robot, sc)
        assert det.check(q)['flags'].sum() == 0
        assert (det.check(q, flags=rtcd.CHECK_CONTAINMENT)['flags'] == 2).all()
        assert (det.check(q, flags=rtcd.CHECK_CONTAINMENT | rtcd.CHECK_TWO_WAY)['flags'] == 2).all()


@pytest.mark.parametrize('name', ['ObsToRobot', 'RobotToObs'])
def test_two_way_is_union_of_directions(setup, panda, name):
    """RTCD_CHECK_TWO_WAY: flags = ObsToRobot | RobotToObs, counts = their sum,
    from either detector kind and through the graph path."""
    robot, scene, (orob, oscene) = setup
    q = scenes.uniform_poses(panda, 700, seed=12)
    o2r = rtcd.Detector(robot.ctx, 'ObsToRobot', robot, scene).check(q, counts=True)
    r2o = rtcd.Detector(robot.ctx, 'RobotToObs', robot, scene).check(q, counts=True)
    det = rtcd.Detector(robot.ctx, name, robot, scene)
    both = det.check(q, counts=True, flags=rtcd.CHECK_TWO_WAY)
    assert np.array_equal(both['flags'], o2r['flags'] | r2o['flags'])
    assert np.array_equal(both['counts'], o2r['counts'] + r2o['counts'])
    assert np.array_equal(det.check(q, flags=rtcd.CHECK_TWO_WAY)['flags'], both['flags'])
    assert np.array_equal(det.check(q, flags=rtcd.CHECK_TWO_WAY | rtcd.CHECK_PLAIN)['flags'], both['flags'])
    ref_h = O.discrete(O.OBS_TO_ROBOT, orob, oscene, q)
    ref_r = O.discrete(O.ROBOT_TO_OBS, orob, oscene, q)
    ok = (ref_h['band'] == 0) & (ref_r['band'] == 0)
    assert np.array_equal(both['flags'][ok], (ref_h['hit'] | ref_r['hit'])[ok])
    assert (both['flags'] > o2r['flags']).sum() + (both['flags'] > r2o['flags']).sum() > 0


def test_graph_with_host_buffers(ctx, panda):
    """RTCD_CHECK_GRAPH with host arrays: the graph holds the staging copies,
    so replays with new pose values (new host arrays of the same size) return
    those poses' flags and counts, equal to the plain host path."""
    mesh = scenes.discrete_small(seed=3)
    robot = rtcd.Robot(ctx, panda)
    scene = rtcd.Scene.from_mesh(ctx, mesh)
    qs = [scenes.uniform_poses(panda, 700, seed=seed) for seed in (0, 1, 2)]
    for kind in ('RobotToObs', 'ObsToRobot'):
        det = rtcd.Detector(ctx, kind, robot, scene)
        refs = [det.check(q, counts=True) for q in qs]
        for q, ref in zip(qs + qs, refs + refs):   # captured on the first call, replayed after
            got = det.check(q, counts=True, flags=rtcd.CHECK_GRAPH)
            assert np.array_equal(got['flags'], ref['flags'])
            assert np.array_equal(got['counts'], ref['counts'])
        for q, ref in zip(qs, refs):
            assert np.array_equal(det.check(q, flags=rtcd.CHECK_GRAPH)['flags'], ref['flags'])
        det.close()


def test_large_triangle_edges_graze_links(ctx, panda):
    """The link-side node test of RobotToObs adds the nine edge-cross axes for
    triangles over 3 cm.  Aim at its boundary: one large triangle per scene
    whose edge passes through, just inside and just outside a link's vertex
    (offsets 0, +-50 um, +-1 mm and tangent-parallel), poses jittered around
    that pose by up to 2 mrad.  Flags and counts equal the FP64 oracle's
    outside the band."""
    robot = rtcd.Robot(ctx, panda)
    rng = np.random.default_rng(21)
    orob = O.Robot(panda)
    checked = hits = 0
    for k in range(8):
        q0 = scenes.uniform_poses(panda, 1, seed=200 + k)[0]
        T = O.fk(panda, q0[None])[0]
        l = 1 + k % 7
        lv = panda['link_verts'][panda['link_vert_off'][l]:panda['link_vert_off'][l + 1]].astype(np.float64)
        Tl = T[l].reshape(3, 4)
        p = lv[rng.integers(len(lv))] @ Tl[:, :3].T + Tl[:, 3]  # a link vertex in the world
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        n = np.cross(d, rng.normal(size=3))
        n /= np.linalg.norm(n)
        off = [0.0, 5e-5, -5e-5, 1e-3, -1e-3][k % 5]
        a = p + off * n - 0.6 * d          # the edge a-b passes off metres from the vertex
        b = p + off * n + 0.6 * d
        c = p + off * n + 0.8 * n + 0.1 * d  # the triangle spans to one side of the edge
        mesh = scenes.Mesh(np.array([a, b, c], np.float32), np.array([[0, 1, 2]], np.uint32),
                           np.array([0, 1], np.uint32))
        sc = rtcd.Scene.from_mesh(ctx, mesh)
        q = (q0[None] + rng.uniform(-2e-3, 2e-3, size=(256, 7))).astype(np.float32)
        q = np.clip(q, panda['lower'], panda['upper'])
        det = rtcd.Detector(ctx, 'RobotToObs', robot, sc)
        ref = O.discrete(O.ROBOT_TO_OBS, orob, O.Scene(mesh), q)
        _compare(det.check(q, counts=True), ref)
        assert np.array_equal(det.check(q)['flags'], det.check(q, counts=True)['flags'])
        checked += int((ref['band'] == 0).sum())
        hits += int(ref['hit'].sum())
        det.close()
        sc.close()
    assert checked > 1000 and hits > 0


def test_plain_path_upstream_shape(setup, panda):
    """The plain path (frames over several streams and host threads, a host
    round trip per frame) equals the batched path for frame sizes and stream
    counts that leave partial frames and partial groups."""
    robot, scene, _ = setup
    q = scenes.uniform_poses(panda, 5000, seed=12)
    base = None
    for fs, ns in ((1024, 4), (1024, 1), (333, 3), (5000, 2)):
        det = rtcd.Detector(robot.ctx, 'RobotToObs', robot, scene, frame_size=fs, plain_streams=ns)
        a = det.check(q, counts=True)
        b = det.check(q, counts=True, flags=rtcd.CHECK_PLAIN)
        assert np.array_equal(a['flags'], b['flags']) and np.array_equal(a['counts'], b['counts'])
        assert det.stats()['work_items'] > 0
        if base is None:
            base = a['flags']
        assert np.array_equal(a['flags'], base)
        det.close()


@pytest.fixture(scope='module')
def dense(ctx, panda):
    mesh = scenes.discrete_dense()  # the graded 428,448-triangle scene
    return rtcd.Robot(ctx, panda), rtcd.Scene.from_mesh(ctx, mesh), O.Robot(panda), O.Scene(mesh)


@pytest.mark.parametrize('name,okind', KINDS)
def test_graded_dense_scene(dense, panda, name, okind):
    """The graded RobotToObs / ObsToRobot workload's scene (64 boxes, 256
    level-3 icospheres, the 100k-triangle noisy sphere: 428,448 triangles) at
    4,096 uniform poses: flags and upstream counts equal the FP64 oracle's
    outside the band, with and without the cull, and the two-way union."""
    robot, scene, orob, osc = dense
    q = scenes.uniform_poses(panda, 4096, seed=0)
    ref = O.discrete(okind, orob, osc, q)
    det = rtcd.Detector(robot.ctx, name, robot, scene)
    _compare(det.check(q, counts=True), ref)
    _compare(det.check(q, counts=True, flags=rtcd.CHECK_NO_CULL), ref)
    assert np.array_equal(det.check(q)['flags'], det.check(q, counts=True)['flags'])
    other = O.discrete(1 - okind, orob, osc, q)
    both = det.check(q, flags=rtcd.CHECK_TWO_WAY)['flags']
    band = (ref['band'] | other['band']).astype(bool)
    assert not ((both != (ref['hit'] | other['hit'])) & ~band).any()
    assert 0.3 < ref['hit'].mean() < 0.95


@pytest.mark.parametrize('name,okind', KINDS)
def test_top_levels_in_shared_memory_agree(dense, panda, name, okind):
    """The fused kernel with the wide tree's top levels staged in shared memory
    (85 nodes: the first four levels; 256: more) gives the same flags and
    counts as without staging."""
    robot, scene, _, _ = dense
    q = scenes.uniform_poses(panda, 2048, seed=5)
    base = rtcd.Detector(robot.ctx, name, robot, scene).check(q, counts=True)
    for top in (85, 256):
        det = rtcd.Detector(robot.ctx, name, robot, scene, top_nodes_shared=top)
        out = det.check(q, counts=True)
        assert np.array_equal(out['flags'], base['flags']) and np.array_equal(out['counts'], base['counts'])
        det.close()


@pytest.mark.parametrize('name,okind', KINDS)
def test_cull_keeps_every_hit_many_obstacles(ctx, panda, name, okind):
    """A scene of 165 obstacles: 90 random boxes and icospheres plus a lattice
    of small boxes.  With the OBB cull, flags and upstream counts equal the
    run without it exactly (no item with a hit is dropped) and the FP64
    oracle's outside the band."""
    base = scenes.random_scene(50, 40, 1, seed=5, box_ext=(0.02, 0.3))
    lattice = [scenes.box_mesh((x, y, z), (0.03, 0.03, 0.03))
               for x in np.linspace(-0.9, 0.9, 5) for y in np.linspace(-0.9, 0.9, 5) for z in (0.2, 0.6, 1.0)]
    verts, tris, off = [base.verts], [base.tris], list(base.obstacle_tri_off)
    nv = len(base.verts)
    for v, t in lattice:
        verts.append(v)
        tris.append(t + nv)
        nv += len(v)
        off.append(off[-1] + len(t))
    mesh = scenes.Mesh(np.concatenate(verts), np.concatenate(tris), np.asarray(off, np.uint32))
    assert mesh.n_obstacles == 165
    scene = rtcd.Scene.from_mesh(ctx, mesh)
    robot = rtcd.Robot(ctx, panda)
    q = scenes.uniform_poses(panda, 2048, seed=17)
    det = rtcd.Detector(ctx, name, robot, scene)
    a = det.check(q, counts=True)
    b = det.check(q, counts=True, flags=rtcd.CHECK_NO_CULL)
    assert np.array_equal(a['flags'], b['flags']) and np.array_equal(a['counts'], b['counts'])
    _compare(a, O.discrete(okind, O.Robot(panda), O.Scene(mesh), q))
    assert a['flags'].any()


def _pinned(a):
    """A page-locked copy of a (torch's pinned allocator), as a numpy view."""
    import torch
    p = torch.empty(a.shape, dtype=torch.float32).pin_memory().numpy()
    p[...] = a
    return p


def test_page_locked_poses_match_pageable(ctx, panda):
    """Host calls whose poses sit in page-locked memory upload them by DMA
    directly, in the direct path and in the graph (captured with the caller's
    array as the copy source): flags and counts equal the pageable calls', a
    pinned array rewritten in place is read afresh on replay, and a switch
    between pinned and pageable arrays re-captures."""
    mesh = scenes.discrete_small(seed=5)
    robot = rtcd.Robot(ctx, panda)
    scene = rtcd.Scene.from_mesh(ctx, mesh)
    qs = [scenes.uniform_poses(panda, 900, seed=seed) for seed in (3, 4)]
    for kind in ('RobotToObs', 'ObsToRobot'):
        det = rtcd.Detector(ctx, kind, robot, scene)
        refs = [det.check(q, counts=True) for q in qs]
        assert any(r['flags'].any() for r in refs)
        pin = _pinned(qs[0])
        for graph in (0, rtcd.CHECK_GRAPH):
            for i in (0, 1, 0, 1):
                pin[...] = qs[i]     # same page-locked array, new values
                got = det.check(pin, counts=True, flags=graph)
                assert np.array_equal(got['flags'], refs[i]['flags'])
                assert np.array_equal(got['counts'], refs[i]['counts'])
                got = det.check(qs[1 - i], counts=True, flags=graph)   # pageable in between
                assert np.array_equal(got['flags'], refs[1 - i]['flags'])
        det.close()
