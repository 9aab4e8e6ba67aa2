"""The reference's own benchmark shelves (models/curobo with the placements of
its scene headers; 15k and 202k triangles): discrete and sweep detectors
against the FP64 oracle, flags outside the 1e-5 m band."""
import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('scene_name', ['simple', 'dense'])
@pytest.mark.parametrize('name,okind', [('ObsToRobot', O.OBS_TO_ROBOT), ('RobotToObs', O.ROBOT_TO_OBS)])
def test_discrete_on_reference_shelves(ctx, panda, scene_name, name, okind):
    mesh = scenes.reference_scene(scene_name)
    robot = rtcd.Robot(ctx, panda)
    sc = rtcd.Scene.from_mesh(ctx, mesh)
    q = scenes.uniform_poses(panda, 384, seed=31)
    out = rtcd.Detector(ctx, name, robot, sc).check(q, counts=True)
    ref = O.discrete(okind, O.Robot(panda), O.Scene(mesh), q)
    ok = ref['band'] == 0
    assert np.array_equal(out['flags'][ok], ref['hit'][ok])
    safe = ref['marg'] == 0
    assert np.array_equal(out['counts'][safe], ref['count'][safe])
    assert 0.1 < ref['hit'].mean() < 0.9


@pytest.mark.parametrize('kind', ['Linear', 'Quadratic'])
def test_sweeps_on_reference_dense_shelf(ctx, panda, kind):
    mesh = scenes.reference_scene('dense')
    sph = scenes.synth_spheres(panda)
    robot = rtcd.Robot(ctx, panda, spheres=sph)
    sc = rtcd.Scene.from_mesh(ctx, mesh)
    counts = 16 if kind == 'Linear' else scenes.log_uniform_counts(48, 8, 16, seed=4)
    q, off = scenes.random_walk_trajectories(panda, 48, counts, seed=4)
    out = rtcd.Detector(ctx, kind, robot, sc).check(q, off, segments=True)
    ref = O.sweep(kind == 'Quadratic', O.Robot(panda, spheres=sph), O.Scene(mesh), q, off)
    ok = ref['traj_band'] == 0
    assert np.array_equal(out['flags'][ok], ref['traj_hit'][ok])
    sok = ref['seg_band'] == 0
    assert np.array_equal(out['seg_flags'][sok], ref['seg_hit'][sok])
