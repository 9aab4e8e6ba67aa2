"""The sweeps under the reference's semantics (RTCD_CHECK_SURFACE: directed
loop edges, an edge hits a piece only when it starts outside the piece and
reaches it; round-capped capsules, flat-capped quadratic pieces without end
spheres) against the FP64 oracle's restatement of the same predicate, on
small cases and on the graded 4,096-trajectory workloads; and the solid
semantics on the graded workloads."""
import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def setup(ctx, panda):
    sph = scenes.synth_spheres(panda, per_link=8, seed=0)
    mesh = scenes.sweep_scene()
    robot = rtcd.Robot(ctx, panda, spheres=sph)
    scene = rtcd.Scene.from_mesh(ctx, mesh)
    return robot, scene, O.Robot(panda, spheres=sph), O.Scene(mesh)


def _cmp(out, ref, counts=False):
    tb = ref['traj_band'].astype(bool)
    m = (out['flags'] != ref['traj_hit']) & ~tb
    assert m.sum() == 0, 'trajectory flag mismatches at %s' % np.nonzero(m)[0][:20]
    if 'seg_flags' in out:
        assert np.array_equal(out['seg_off'], ref['seg_off'])
        sb = ref['seg_band'].astype(bool)
        ms = (out['seg_flags'] != ref['seg_hit']) & ~sb
        assert ms.sum() == 0, 'segment flag mismatches at %s' % np.nonzero(ms)[0][:20]
    if counts:
        safe = ~ref['traj_marg'].astype(bool)
        mc = (out['counts'] != ref['traj_count']) & safe
        assert mc.sum() == 0, 'count mismatches at %s' % np.nonzero(mc)[0][:20]


def test_surface_linear_parity(setup, panda):
    robot, scene, orob, osc = setup
    q, off = scenes.random_walk_trajectories(panda, 256, 32, seed=0)
    ref = O.sweep(False, orob, osc, q, off, surface=True)
    det = rtcd.Detector(robot.ctx, 'Linear', robot, scene)
    _cmp(det.check(q, off, segments=True, surface=True), ref)
    _cmp(det.check(q, off, counts=True, segments=True, surface=True), ref, counts=True)
    _cmp(det.check(q, off, surface=True), ref)
    assert 0.05 < ref['traj_hit'].mean()


def test_surface_quadratic_parity_uneven(setup, panda):
    robot, scene, orob, osc = setup
    n_wp = scenes.log_uniform_counts(192, 8, 64, seed=1)
    q, off = scenes.random_walk_trajectories(panda, 192, n_wp, seed=1)
    ref = O.sweep(True, orob, osc, q, off, surface=True)
    det = rtcd.Detector(robot.ctx, 'Quadratic', robot, scene)
    _cmp(det.check(q, off, segments=True, surface=True), ref)
    _cmp(det.check(q, off, counts=True, segments=True, surface=True), ref, counts=True)
    # surface semantics carry no end spheres: NO_ENDPOINTS changes nothing
    a = det.check(q, off, segments=True, surface=True, flags=rtcd.CHECK_NO_ENDPOINTS)
    _cmp(a, ref)


def test_surface_hits_are_solid_hits(setup, panda):
    """Per segment the entering-ray hits are a subset of the solid hits."""
    robot, scene, _, _ = setup
    for kind in ('Linear', 'Quadratic'):
        n_wp = scenes.log_uniform_counts(512, 8, 64, seed=7)
        q, off = scenes.random_walk_trajectories(panda, 512, n_wp, seed=7)
        det = rtcd.Detector(robot.ctx, kind, robot, scene)
        a = det.check(q, off, segments=True, flags=rtcd.CHECK_NO_ENDPOINTS)
        b = det.check(q, off, segments=True, surface=True)
        assert np.array_equal(a['seg_off'], b['seg_off'])
        assert np.all(b['seg_flags'] <= a['seg_flags'])
        assert b['seg_flags'].sum() > 0


def test_surface_graph_replay_and_server(setup, panda):
    robot, scene, _, _ = setup
    import torch
    n_wp = scenes.log_uniform_counts(128, 8, 64, seed=9)
    q, off = scenes.random_walk_trajectories(panda, 128, n_wp, seed=9)
    det = rtcd.Detector(robot.ctx, 'Quadratic', robot, scene)
    want = det.check(q, off, surface=True)['flags']
    qd = torch.from_numpy(q).cuda()
    fl = torch.zeros(len(off) - 1, dtype=torch.uint8, device='cuda')
    for _ in range(3):
        fl.zero_()
        det.check_device(qd, len(off) - 1, fl, traj_off=off, flags=rtcd.CHECK_GRAPH | rtcd.CHECK_SURFACE)
        torch.cuda.synchronize()
        assert np.array_equal(fl.cpu().numpy(), want)
    srv = rtcd.Server(robot.ctx, slots=2)
    t = srv.submit(det, q, off, surface=True)
    assert np.array_equal(srv.wait(t)['flags'], want)
    srv.close()


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
@pytest.mark.parametrize('surface', [False, True])
def test_graded_sweep_workloads(setup, panda, kind, surface):
    """The graded workloads at full size: 4,096 trajectories of 32 waypoints
    (linear) and of 8-64 waypoints, log-uniform (quadratic), random walks
    N(0, 0.1) rad; 64 spheres; the 49,744-triangle shelf-and-sphere scene.
    Trajectory and segment flags equal the oracle's outside the band."""
    robot, scene, orob, osc = setup
    quad = kind == 'Quadratic'
    if quad:
        n_wp = scenes.log_uniform_counts(4096, 8, 64, seed=0)
        q, off = scenes.random_walk_trajectories(panda, 4096, n_wp, seed=0)
    else:
        q, off = scenes.random_walk_trajectories(panda, 4096, 32, seed=0)
    ref = O.sweep(quad, orob, osc, q, off, surface=surface)
    det = rtcd.Detector(robot.ctx, kind, robot, scene)
    out = det.check(q, off, segments=True, surface=surface)
    _cmp(out, ref)
    assert ref['seg_band'].mean() < 0.01
