"""Robot input at run time (host only, no GPU): the library's URDF chain
reader reproduces the reference's generated Panda masks, folds fixed joints,
handles other joint axes, and rejects what it does not support; the OBJ
loader deduplicates vertices as the reference's loader does."""
import json
import os

import numpy as np
import pytest

from rtcollisiondetection_b200 import rtcd
from rtcollisiondetection_b200.data.make_panda import dedupe_mesh, parse_obj

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _urdf(chain, extra_joints=(), drop_limits=False):
    out = ['<?xml version="1.0"?>', '<!-- test robot -->', '<robot name="r">']
    for l in chain['links']:
        if l['mesh']:
            out.append('<link name="%s"><visual><origin xyz="0 0 0" rpy="0 0 0"/><geometry>'
                       '<mesh filename="%s"/></geometry></visual></link>' % (l['name'], l['mesh']))
        else:
            out.append('<link name="%s"/>' % l['name'])
    for j in list(chain['joints']) + list(extra_joints):
        lim = '' if drop_limits or j['lower'] is None else \
            '<limit effort="1" lower="%s" upper="%s" velocity="1"/>' % (j['lower'], j['upper'])
        out.append('<joint name="%s" type="%s"><parent link="%s"/><child link="%s"/>'
                   '<origin rpy="%s" xyz="%s"/><axis xyz="%s"/>%s</joint>'
                   % (j['name'], j['type'], j['parent'], j['child'], j['rpy'], j['xyz'], j['axis'], lim))
    out.append('</robot>')
    return '\n'.join(out)


def test_urdf_masks_equal_reference_header():
    """The reference's generated panda.h, rebuilt from the Panda's URDF chain."""
    chain = json.load(open(os.path.join(GOLDEN, 'panda_chain.json')))
    hdr = json.load(open(os.path.join(GOLDEN, 'panda_header.json')))
    c = rtcd.urdf_chain(_urdf(chain))
    assert c['dof'] == 7 and len(c['link_names']) == 8
    for hk, ck in (('cosMask', 'cos_mask'), ('sinMask', 'sin_mask'), ('oneMask', 'one_mask')):
        assert np.array_equal(np.array(hdr[hk], np.float32).reshape(7, 12), c[ck]), hk
    assert np.array_equal(np.array(hdr['baseT'], np.float32), c['base_tf'])
    assert np.array_equal(np.array(hdr['lowerBound'], np.float32), c['lower'])
    assert np.array_equal(np.array(hdr['upperBound'], np.float32), c['upper'])
    assert c['link_meshes'][3] == 'merged_meshes/panda_link3_visual.obj'


def _fk(c, q):
    T = np.eye(4)
    out = [T]
    for i in range(c['dof']):
        L = np.cos(q[i]) * c['cos_mask'][i] + np.sin(q[i]) * c['sin_mask'][i] + c['one_mask'][i]
        M = np.eye(4)
        M[:3, :] = L.reshape(3, 4)
        T = T @ M
        out.append(T)
    return out


def _rot(axis, t):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(t) * K + (1 - np.cos(t)) * K @ K


def _origin(rpy, xyz):
    r, p, y = rpy
    Rx = _rot([1, 0, 0], r)
    Ry = _rot([0, 1, 0], p)
    Rz = _rot([0, 0, 1], y)
    M = np.eye(4)
    M[:3, :3] = Rz @ Ry @ Rx
    M[:3, 3] = xyz
    return M


def test_urdf_fixed_joints_and_general_axes():
    """A chain with a fixed joint between two revolute joints and tilted axes:
    the masks reproduce origin * fixed * origin * Rot(axis, q) exactly."""
    chain = {'links': [{'name': n, 'mesh': ''} for n in ('a', 'b', 'c', 'd')], 'joints': [
        {'name': 'j1', 'type': 'revolute', 'parent': 'a', 'child': 'b', 'rpy': '0.3 -0.2 0.1',
         'xyz': '0.1 0 0.2', 'axis': '0 1 1', 'lower': '-1', 'upper': '1'},
        {'name': 'f', 'type': 'fixed', 'parent': 'b', 'child': 'c', 'rpy': '0 0.7 0', 'xyz': '0 0.05 0',
         'axis': '1 0 0', 'lower': None, 'upper': None},
        {'name': 'j2', 'type': 'continuous', 'parent': 'c', 'child': 'd', 'rpy': '0 0 0.4', 'xyz': '0.2 0 0',
         'axis': '1 0 0', 'lower': None, 'upper': None}]}
    c = rtcd.urdf_chain(_urdf(chain))
    assert c['dof'] == 2 and c['link_names'] == ['a', 'b', 'd']
    assert np.allclose(c['lower'], [-1, -np.pi]) and np.allclose(c['upper'], [1, np.pi])
    q = [0.7, -1.3]
    T = _fk(c, q)
    J1 = _origin([0.3, -0.2, 0.1], [0.1, 0, 0.2])
    R1 = np.eye(4); R1[:3, :3] = _rot([0, 1, 1], q[0])
    F = _origin([0, 0.7, 0], [0, 0.05, 0])
    J2 = _origin([0, 0, 0.4], [0.2, 0, 0])
    R2 = np.eye(4); R2[:3, :3] = _rot([1, 0, 0], q[1])
    assert np.allclose(T[1], J1 @ R1, atol=1e-6)
    assert np.allclose(T[2], J1 @ R1 @ F @ J2 @ R2, atol=1e-6)


@pytest.mark.parametrize('bad', ['branch', 'prismatic', 'no_limits', 'malformed', 'not_robot'])
def test_urdf_rejects_unsupported(bad):
    chain = json.load(open(os.path.join(GOLDEN, 'panda_chain.json')))
    if bad == 'branch':
        text = _urdf(chain, extra_joints=[dict(chain['joints'][0], name='x', child='extra')])
        text = text.replace('</robot>', '<link name="extra"/></robot>')
    elif bad == 'prismatic':
        chain['joints'][2]['type'] = 'prismatic'
        text = _urdf(chain)
    elif bad == 'no_limits':
        text = _urdf(chain, drop_limits=True)
    elif bad == 'malformed':
        text = _urdf(chain)[:-40]
    else:
        text = '<robots></robots>'
    with pytest.raises(rtcd.RTCDError) as e:
        rtcd.urdf_chain(text)
    assert e.value.status == 1


def test_obj_loader_matches_upstream_dedupe(tmp_path):
    """Quads, a pentagon, repeated positions under other indices, negative
    indices and texture/normal refs: same vertices and triangles as the
    reference-style loader restated in make_panda.py."""
    p = tmp_path / 'm.obj'
    p.write_text('\n'.join([
        '# test', 'v 0 0 0', 'v 1 0 0', 'v 1 1 0', 'v 0 1 0', 'v 0 0 1', 'v 1 0 0', 'v 0.5 0.5 2',
        'vt 0 0', 'vn 0 0 1',
        'f 1/1/1 2/1/1 3/1/1 4/1/1', 'f 1 5 6', 'f -1 -2 -3', 'f 1 2 7 4 5', 'usemtl x', 's off']) + '\n')
    v, t = rtcd.obj_load(str(p))
    raw, faces = parse_obj(str(p))
    rv, rt, _ = dedupe_mesh(raw, faces)
    assert np.array_equal(v, rv) and np.array_equal(t, rt)
    assert len(v) == 6  # vertex 6 repeats vertex 2's position
    with pytest.raises(rtcd.RTCDError):
        rtcd.obj_load(str(tmp_path / 'missing.obj'))


def test_halton_samples_restate_reference_arithmetic():
    """Host only: the reference's float radical inverse, scaled into the bounds."""
    lo = np.array([-1.0, 0.0, 2.0], np.float32)
    hi = np.array([1.0, 0.5, 3.0], np.float32)
    got = rtcd.halton_samples(200, lo, hi, skip=2)
    primes = [5, 7, 11]

    def radical(n, b):
        hn, n0, f = np.float32(0), n, np.float32(1) / np.float32(b)
        while n0 > 0:
            n1 = np.float32(n0 // b)
            r = n0 - int(n1 * np.float32(b))
            hn = np.float32(hn + f * np.float32(r))
            f = np.float32(f / np.float32(b))
            n0 = int(n1)
        return hn
    ref = np.array([[np.float32(radical(i, primes[d]) * (hi[d] - lo[d]) + lo[d]) for d in range(3)]
                    for i in range(200)], np.float32)
    assert np.array_equal(got, ref)
    assert got[0].tolist() == lo.tolist()
    with pytest.raises(rtcd.RTCDError):
        rtcd.halton_samples(4, np.zeros(20), np.ones(20), skip=10)
