"""Regenerate the golden fixtures in this folder from the upstream repository.

Run where the upstream RTCollisionDetection checkout is available:
    python tests/golden/make_golden.py <upstream root>

Writes
* ``panda_header.json`` - the cos/sin/one masks, base transform and joint
  limits as literal numbers from ``RTCD/Robot/models/panda.h:7-44``; the test
  suite checks that masks derived from the URDF reproduce them.
* ``quad_weights.npz``  - the shipped least-squares quadratic B-spline fit
  matrices ``RTCD/data/weights/quad/normal/{nC}_{nT}.txt`` (row-major nC x nT),
  the known answers for the on-device fit weights.
* ``panda_mesh_stats.json`` - per-link vertex/triangle/unique-edge counts of
  the merged visual meshes, counted here with a direct text scan of the OBJ
  files (independent of the package loader).
* ``panda_chain.json`` - the kinematic chain of the Panda URDF
  (``models/franka_description/modified_panda.urdf``): per joint its parent,
  child, type, origin (rpy, xyz), axis and limits, per link its visual mesh
  file name; the tests rebuild a URDF from it for the C++ URDF reader.
"""
import json
import os
import re
import sys
import glob
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def header_arrays(path):
    src = open(path).read()
    out = {}
    for name in ('baseT', 'lowerBound', 'upperBound', 'sinMask', 'cosMask', 'oneMask'):
        m = re.search(name + r'[^{;]*\{([^}]*)\}', src)
        nums = re.findall(r'-?\d+\.?\d*(?:e-?\d+)?', m.group(1))
        out[name] = [float(x) for x in nums]
    return out


def mesh_stats(root):
    stats = []
    for li in range(8):
        p = os.path.join(root, 'models/franka_description/merged_meshes/panda_link%d_visual.obj' % li)
        pos, faces = [], []
        for line in open(p):
            if line.startswith('v '):
                pos.append(tuple(np.float32(float(x)) for x in line.split()[1:4]))
            elif line.startswith('f '):
                faces.append([int(t.split('/')[0]) - 1 for t in line.split()[1:]])
        uniq = {}
        for v in pos:
            uniq.setdefault(v, len(uniq))
        edges = set()
        for f in faces:
            g = [uniq[pos[i]] for i in f]
            for a, b in ((g[0], g[1]), (g[1], g[2]), (g[2], g[0])):
                edges.add((min(a, b), max(a, b)))
        stats.append({'verts': len(uniq), 'tris': len(faces), 'edges': len(edges)})
    return stats


def panda_chain(urdf):
    import xml.etree.ElementTree as ET
    r = ET.parse(urdf).getroot()
    links = []
    for l in r.findall('link'):
        m = l.find('visual/geometry/mesh')
        links.append({'name': l.get('name'), 'mesh': m.get('filename') if m is not None else ''})
    joints = []
    for j in r.findall('joint'):
        o = j.find('origin')
        lim = j.find('limit')
        ax = j.find('axis')
        joints.append({'name': j.get('name'), 'type': j.get('type'), 'parent': j.find('parent').get('link'),
                       'child': j.find('child').get('link'),
                       'rpy': o.get('rpy', '0 0 0') if o is not None else '0 0 0',
                       'xyz': o.get('xyz', '0 0 0') if o is not None else '0 0 0',
                       'axis': ax.get('xyz') if ax is not None else '1 0 0',
                       'lower': lim.get('lower') if lim is not None else None,
                       'upper': lim.get('upper') if lim is not None else None})
    return {'links': links, 'joints': joints}


def main(root):
    hdr = header_arrays(os.path.join(root, 'RTCD/Robot/models/panda.h'))
    json.dump(hdr, open(os.path.join(HERE, 'panda_header.json'), 'w'), indent=1)
    w = {}
    for f in sorted(glob.glob(os.path.join(root, 'RTCD/data/weights/quad/normal/*.txt'))):
        key = os.path.basename(f)[:-4]
        nc, nt = map(int, key.split('_'))
        w['w_' + key] = np.loadtxt(f, dtype=np.float32).reshape(nc, nt)
    np.savez_compressed(os.path.join(HERE, 'quad_weights.npz'), **w)
    json.dump(mesh_stats(root), open(os.path.join(HERE, 'panda_mesh_stats.json'), 'w'), indent=1)
    json.dump(panda_chain(os.path.join(root, 'models/franka_description/modified_panda.urdf')),
              open(os.path.join(HERE, 'panda_chain.json'), 'w'), indent=1)


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: python tests/golden/make_golden.py <upstream root>')
    main(sys.argv[1])
