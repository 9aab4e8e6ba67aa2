"""Launch shapes and the autotuner: every traversal shape returns the same
flags; the autotuner keeps one of the offered shapes."""
import numpy as np
import pytest

from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('kind', ['RobotToObs', 'ObsToRobot', 'Linear', 'Quadratic'])
def test_shapes_agree_and_autotune(ctx, panda, kind):
    import torch
    sph = scenes.synth_spheres(panda)
    robot = rtcd.Robot(ctx, panda, spheres=sph)
    scene = rtcd.Scene.from_mesh(ctx, scenes.discrete_small() if kind in ('RobotToObs', 'ObsToRobot')
                                 else scenes.sweep_scene())
    if kind in ('Linear', 'Quadratic'):
        q, off = scenes.random_walk_trajectories(panda, 96, scenes.log_uniform_counts(96, 8, 40, seed=4), seed=4)
        n = 96
    else:
        q, off, n = scenes.uniform_poses(panda, 700, seed=4), None, 700
    ref = rtcd.Detector(ctx, kind, robot, scene).check(q, off, counts=True)
    for threads in (64, 128, 256):
        for per_sm in (1, 0):
            det = rtcd.Detector(ctx, kind, robot, scene, traverse_threads=threads, traverse_blocks_per_sm=per_sm)
            out = det.check(q, off, counts=True)
            assert np.array_equal(out['flags'], ref['flags']), (threads, per_sm)
            assert np.array_equal(out['counts'], ref['counts']), (threads, per_sm)
    det = rtcd.Detector(ctx, kind, robot, scene)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        qd = torch.from_numpy(q).cuda()
        best = det.autotune(qd, n, off, stream=s.cuda_stream)
    assert best['traverse_threads'] in (64, 128, 256) and best['traverse_blocks_per_sm'] >= 1
    assert best['traverse_ms'] > 0
    assert np.array_equal(det.check(q, off)['flags'], ref['flags'])


def test_bad_launch_shape_rejected(ctx, panda):
    robot = rtcd.Robot(ctx, panda)
    scene = rtcd.Scene.from_mesh(ctx, scenes.discrete_small())
    with pytest.raises(rtcd.RTCDError):
        rtcd.Detector(ctx, 'RobotToObs', robot, scene, traverse_threads=96)
