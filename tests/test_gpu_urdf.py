"""A robot loaded at run time - URDF text through the library's chain reader,
link meshes through its OBJ loader - checks exactly like the prepared Panda
model it describes."""
import json
import os

import numpy as np
import pytest

from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def test_runtime_robot_equals_prepared_model(ctx, panda, small_scene, tmp_path):
    chain = json.load(open(os.path.join(GOLDEN, 'panda_chain.json')))
    # the Panda's link meshes as OBJ files, and a URDF that names them
    for li, l in enumerate(chain['links']):
        v = panda['link_verts'][panda['link_vert_off'][li]:panda['link_vert_off'][li + 1]]
        t = panda['link_tris'][panda['link_tri_off'][li]:panda['link_tri_off'][li + 1]]
        path = tmp_path / ('link%d.obj' % li)
        with open(path, 'w') as fh:
            fh.writelines('v %.9g %.9g %.9g\n' % tuple(x) for x in v)
            fh.writelines('f %d %d %d\n' % tuple(x + 1) for x in t)
        l['mesh'] = path.name
    parts = ['<robot name="panda">']
    parts += ['<link name="%s"><visual><geometry><mesh filename="%s"/></geometry></visual></link>'
              % (l['name'], l['mesh']) for l in chain['links']]
    parts += ['<joint name="%s" type="%s"><parent link="%s"/><child link="%s"/><origin rpy="%s" xyz="%s"/>'
              '<axis xyz="%s"/><limit lower="%s" upper="%s"/></joint>'
              % (j['name'], j['type'], j['parent'], j['child'], j['rpy'], j['xyz'], j['axis'], j['lower'], j['upper'])
              for j in chain['joints']]
    parts.append('</robot>')
    model = rtcd.model_from_urdf('\n'.join(parts), str(tmp_path))
    for k in ('link_verts', 'link_tris', 'link_vert_off', 'link_tri_off', 'cos_mask', 'sin_mask', 'one_mask'):
        assert np.array_equal(np.asarray(model[k]).ravel(), np.asarray(panda[k]).ravel()), k
    sc = rtcd.Scene.from_mesh(ctx, small_scene)
    q = scenes.uniform_poses(panda, 500, seed=17)
    a = rtcd.Robot(ctx, model, edges=False)      # unique edges extracted by the library
    b = rtcd.Robot(ctx, panda)
    for kind in ('ObsToRobot', 'RobotToObs'):
        ra = rtcd.Detector(ctx, kind, a, sc).check(q, counts=True)
        rb = rtcd.Detector(ctx, kind, b, sc).check(q, counts=True)
        assert np.array_equal(ra['flags'], rb['flags']) and np.array_equal(ra['counts'], rb['counts'])
