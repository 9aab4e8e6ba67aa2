"""Generate ``panda.npz``: the Franka Panda robot model as flat arrays.

This is a data-preparation script, run once where the upstream model files are
available.  It reads the URDF (joint origins, axes, limits), the eight merged
visual link meshes and the per-link sphere files of
``models/franka_description`` and writes every array the detector needs:

* link meshes, deduplicated the way the upstream loader does it
  (``RTCD/Meshes/mesh.h:218-231``: a vertex is identified by its exact float
  position, first occurrence wins, faces visited in file order), triangles as
  indices into the per-link vertex list, and the unique undirected edges in
  first-seen orientation (``RTCD/Meshes/mesh.h:200-216``);
* the per-joint cos/sin/one masks of the local transform
  ``L_i(q) = cos(q) C_i + sin(q) S_i + O_i`` derived from the URDF joint
  origin (rpy, xyz) and a z rotation axis (the form of
  ``RTCD/Robot/models/panda.h:16-44``), the identity base transform and the
  joint limits;
* the 62 shipped link spheres (``x y z r`` per line).

Usage:  python make_panda.py <franka_description dir> <out.npz>
"""
import sys
import os
import xml.etree.ElementTree as ET
import numpy as np


def parse_obj(path):
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            if line.startswith('v '):
                verts.append([float(x) for x in line.split()[1:4]])
            elif line.startswith('f '):
                idx = [int(tok.split('/')[0]) for tok in line.split()[1:]]
                idx = [i - 1 if i > 0 else len(verts) + i for i in idx]
                for k in range(1, len(idx) - 1):          # fan triangulation
                    faces.append((idx[0], idx[k], idx[k + 1]))
    return np.asarray(verts, dtype=np.float32), faces


def dedupe_mesh(raw_verts, faces):
    known = {}
    verts, tris, edges, seen = [], [], [], set()

    def vid(v):
        key = (float(v[0]), float(v[1]), float(v[2]))
        if key not in known:
            known[key] = len(verts)
            verts.append(v)
        return known[key]

    for f in faces:
        g = [vid(raw_verts[i]) for i in f]
        tris.append(g)
        for a, b in ((g[0], g[1]), (g[1], g[2]), (g[2], g[0])):
            k = (min(a, b), max(a, b))
            if k not in seen:
                seen.add(k)
                edges.append((a, b))
    return (np.asarray(verts, dtype=np.float32), np.asarray(tris, dtype=np.uint32),
            np.asarray(edges, dtype=np.uint32))


def rpy_matrix(r, p, y):
    cr, sr, cp, sp, cy, sy = np.cos(r), np.sin(r), np.cos(p), np.sin(p), np.cos(y), np.sin(y)
    rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return rz @ ry @ rx


def joint_masks(rpy, xyz):
    """cos/sin/one masks (3x4 row-major) of origin(rpy, xyz) * Rz(q)."""
    R = rpy_matrix(*rpy)
    C = np.zeros((3, 4)); S = np.zeros((3, 4)); O = np.zeros((3, 4))
    C[:, :3] = R @ np.diag([1.0, 1.0, 0.0])
    S[:, :3] = R @ np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    O[:, :3] = R @ np.diag([0.0, 0.0, 1.0])
    O[:, 3] = xyz
    out = []
    for M in (C, S, O):
        M = np.where(np.abs(M) < 1e-9, 0.0, M)     # rpy of +-pi/2 leaves ~1e-12 residues
        out.append(M.astype(np.float32).reshape(12))
    return out


def main(root, out):
    tree = ET.parse(os.path.join(root, 'modified_panda.urdf')).getroot()
    links = [l.get('name') for l in tree.findall('link')]
    joints = [j for j in tree.findall('joint') if j.get('type') == 'revolute']
    cos_m, sin_m, one_m, lower, upper = [], [], [], [], []
    for j in joints:
        o = j.find('origin')
        rpy = [float(x) for x in o.get('rpy').split()]
        xyz = [float(x) for x in o.get('xyz').split()]
        axis = [float(x) for x in j.find('axis').get('xyz').split()]
        assert axis == [0.0, 0.0, 1.0], 'only z-axis revolute joints are modelled'
        c, s, one = joint_masks(rpy, xyz)
        cos_m.append(c); sin_m.append(s); one_m.append(one)
        lim = j.find('limit')
        lower.append(float(lim.get('lower'))); upper.append(float(lim.get('upper')))

    V, T, E = [], [], []
    voff, toff, eoff = [0], [0], [0]
    sc, sr, sl = [], [], []
    for li, name in enumerate(links):
        raw, faces = parse_obj(os.path.join(root, 'merged_meshes', name + '_visual.obj'))
        v, t, e = dedupe_mesh(raw, faces)
        V.append(v); T.append(t); E.append(e)
        voff.append(voff[-1] + len(v)); toff.append(toff[-1] + len(t)); eoff.append(eoff[-1] + len(e))
        sph = np.loadtxt(os.path.join(root, 'spheres', name + '.txt'), dtype=np.float64).reshape(-1, 4)
        sc.append(sph[:, :3]); sr.append(sph[:, 3]); sl += [li] * len(sph)

    np.savez_compressed(
        out,
        link_verts=np.concatenate(V), link_vert_off=np.asarray(voff, np.uint32),
        link_tris=np.concatenate(T), link_tri_off=np.asarray(toff, np.uint32),
        link_edges=np.concatenate(E), link_edge_off=np.asarray(eoff, np.uint32),
        cos_mask=np.stack(cos_m), sin_mask=np.stack(sin_m), one_mask=np.stack(one_m),
        base_tf=np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32),
        lower=np.asarray(lower, np.float32), upper=np.asarray(upper, np.float32),
        sphere_centers=np.concatenate(sc).astype(np.float32),
        sphere_radii=np.concatenate(sr).astype(np.float32),
        sphere_links=np.asarray(sl, np.uint32))
    print('links', len(links), 'verts', voff[-1], 'tris', toff[-1], 'edges', eoff[-1], 'spheres', len(sl))


if __name__ == '__main__':
    main(sys.argv[1], sys.argv[2])
