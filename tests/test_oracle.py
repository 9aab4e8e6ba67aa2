"""The FP64 oracle, pinned to the upstream golden data and to independent
restatements (no GPU)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def test_fit_weights_match_shipped_tables():
    """W = pinv(B) reproduces every shipped RTCD/data/weights/quad/normal table."""
    g = np.load(os.path.join(GOLDEN, 'quad_weights.npz'))
    assert len(g.files) >= 18
    for k in g.files:
        nc, nt = map(int, k[2:].split('_'))
        W = O.fit_weights(nc, nt)
        assert np.abs(W - g[k]).max() < 2e-6, k


def test_urdf_masks_match_upstream_header(panda):
    """Masks derived from the URDF equal RTCD/Robot/models/panda.h:16-44."""
    h = json.load(open(os.path.join(GOLDEN, 'panda_header.json')))
    for hk, pk in (('cosMask', 'cos_mask'), ('sinMask', 'sin_mask'), ('oneMask', 'one_mask')):
        assert np.array_equal(np.array(h[hk], np.float32).reshape(7, 12), panda[pk])
    assert np.array_equal(np.array(h['baseT'], np.float32), panda['base_tf'])
    assert np.array_equal(np.array(h['lowerBound'], np.float32), panda['lower'])
    assert np.array_equal(np.array(h['upperBound'], np.float32), panda['upper'])


def test_mesh_loader_counts(panda):
    stats = json.load(open(os.path.join(GOLDEN, 'panda_mesh_stats.json')))
    assert np.array_equal(np.diff(panda['link_vert_off']), [s['verts'] for s in stats])
    assert np.array_equal(np.diff(panda['link_tri_off']), [s['tris'] for s in stats])
    assert np.array_equal(np.diff(panda['link_edge_off']), [s['edges'] for s in stats])
    assert panda['link_edge_off'][-1] == 35991


def test_unique_edges_first_seen_orientation(panda):
    to, eo = panda['link_tri_off'], panda['link_edge_off']
    for l in range(8):
        e = O.unique_edges(panda['link_tris'][to[l]:to[l + 1]])
        assert np.array_equal(e, panda['link_edges'][eo[l]:eo[l + 1]])
    # tiny hand case: two triangles sharing an edge (given in opposite orientation)
    e = O.unique_edges(np.array([[0, 1, 2], [2, 1, 3]], np.uint32))
    assert e.tolist() == [[0, 1], [1, 2], [2, 0], [1, 3], [3, 2]]


def _fk_numpy(panda, q):
    T = np.array(panda['base_tf'], np.float64).reshape(3, 4)
    out = [T]
    for i, qi in enumerate(q):
        L = (np.cos(qi) * panda['cos_mask'][i] + np.sin(qi) * panda['sin_mask'][i] +
             panda['one_mask'][i]).astype(np.float64).reshape(3, 4)
        M = np.eye(4)
        M[:3] = out[-1]
        N = np.eye(4)
        N[:3] = L
        out.append((M @ N)[:3])
    return np.stack(out)


def test_fk_matches_matrix_chain(panda):
    q = scenes.uniform_poses(panda, 16, seed=1)
    T = O.fk(panda, q)
    for i in range(16):
        assert np.abs(T[i].reshape(8, 3, 4) - _fk_numpy(panda, q[i].astype(np.float64))).max() < 1e-12


def test_fk_zero_pose_link_origins(panda):
    """At q = 0 the Panda's link origins sit at the URDF joint offsets."""
    T = O.fk(panda, np.zeros((1, 7), np.float32))[0].reshape(8, 3, 4)
    assert np.allclose(T[1][:, 3], [0, 0, 0.333], atol=1e-7)
    assert np.allclose(T[3][:, 3], [0, 0, 0.649], atol=1e-6)
    assert np.allclose(T[4][:, 3], [0.0825, 0, 0.649], atol=1e-6)
    assert np.allclose(T[5][:, 3], [0, 0, 1.033], atol=1e-6)
    assert np.allclose(T[7][:, 3], [0.088, 0, 1.033], atol=1e-6)


def test_seg_tri_cases():
    a, b, c = [0, 0, 0], [1, 0, 0], [0, 1, 0]
    assert O.seg_tri([0.2, 0.2, -1], [0.2, 0.2, 1], a, b, c)[0]
    hit, m = O.seg_tri([0.2, 0.2, -1], [0.2, 0.2, 1], a, b, c)
    assert abs(m - 0.2) < 1e-12                     # margin: distance to the nearest edge line
    assert not O.seg_tri([0.2, 0.2, 0.1], [0.2, 0.2, 1], a, b, c)[0]
    miss, d = O.seg_tri([0.2, 0.2, 0.1], [0.2, 0.2, 1], a, b, c)
    assert abs(d - 0.1) < 1e-12
    assert not O.seg_tri([2, 2, -1], [2, 2, 1], a, b, c)[0]
    # touching at a vertex counts as a hit with zero margin
    hit, m = O.seg_tri([0, 0, -1], [0, 0, 1], a, b, c)
    assert hit and m == 0.0
    # coplanar crossing
    hit, m = O.seg_tri([-1, 0.3, 0], [2, 0.3, 0], a, b, c)
    assert hit and m == 0.0


def test_seg_seg_known_answers():
    assert abs(O.seg_seg([0, 0, 0], [1, 0, 0], [0, 1, 1], [1, 1, 1]) - 2 ** 0.5) < 1e-12
    assert O.seg_seg([0, 0, 0], [1, 0, 0], [0.5, -1, 0], [0.5, 1, 0]) == 0.0
    assert abs(O.seg_seg([0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 0]) - 1.0) < 1e-12


def test_seg_quad_against_dense_sampling():
    rng = np.random.default_rng(4)
    for _ in range(200):
        p, q, b0, b1, b2 = rng.uniform(-1, 1, size=(5, 3))
        d = O.seg_quad(p, q, b0, b1, b2)
        u = np.linspace(0, 1, 4001)[:, None]
        C = b0 * (1 - u) ** 2 + 2 * b1 * u * (1 - u) + b2 * u ** 2
        dvec = q - p
        s = np.clip(((C - p) @ dvec) / (dvec @ dvec), 0, 1)[:, None]
        ref = np.linalg.norm(C - (p + s * dvec), axis=1).min()
        assert d <= ref + 1e-12 and d > ref - 1e-5


def test_canonical_lbvh_is_a_valid_tree():
    m = scenes.discrete_small()
    P = m.verts[m.tris]
    lo, hi = P.min(1), P.max(1)
    codes, perm, child, nlo, nhi = O.lbvh(lo, hi)
    n = len(lo)
    assert np.all(np.diff(codes.astype(np.int64)) >= 0)
    assert sorted(perm.tolist()) == list(range(n))
    seen_leaf, seen_int = np.zeros(n, int), np.zeros(n - 1, int)
    for c in child.ravel():
        if c < 0:
            seen_leaf[~c] += 1
        else:
            seen_int[c] += 1
    assert np.all(seen_leaf == 1) and seen_int[0] == 0 and np.all(seen_int[1:] == 1)
    for i in range(n - 1):
        for c in child[i]:
            clo, chi = (lo[perm[~c]], hi[perm[~c]]) if c < 0 else (nlo[c], nhi[c])
            assert np.all(nlo[i] <= clo) and np.all(nhi[i] >= chi)


def _seg_tri_numpy(P, Q, A, B, Cc):
    """Vectorised closed segment-triangle crossing test (signed volumes), an
    independent restatement for the brute-force check."""
    n = np.cross(B - A, Cc - A)
    dp = np.einsum('...k,...k->...', n, P - A)
    dq = np.einsum('...k,...k->...', n, Q - A)
    cross_plane = ~(((dp > 0) & (dq > 0)) | ((dp < 0) & (dq < 0)))
    d = Q - P
    v1 = np.einsum('...k,...k->...', d, np.cross(A - P, B - P))
    v2 = np.einsum('...k,...k->...', d, np.cross(B - P, Cc - P))
    v3 = np.einsum('...k,...k->...', d, np.cross(Cc - P, A - P))
    same = ((v1 >= 0) & (v2 >= 0) & (v3 >= 0)) | ((v1 <= 0) & (v2 <= 0) & (v3 <= 0))
    return cross_plane & same


def test_discrete_oracle_matches_brute_force(panda):
    """Tiny scene: the BVH-accelerated oracle equals an all-pairs loop."""
    mesh = scenes.random_scene(3, 3, 0, seed=3)
    q = scenes.uniform_poses(panda, 12, seed=2)
    R, S = O.Robot(panda), O.Scene(mesh)
    T = O.fk(panda, q)
    sv = mesh.verts.astype(np.float64)
    tri = sv[mesh.tris]                          # k x 3 x 3
    sedge = sv[S.edges]                          # m x 2 x 3
    checked = 0
    for kind in (O.OBS_TO_ROBOT, O.ROBOT_TO_OBS):
        out = O.discrete(kind, R, S, q)
        for i in range(len(q)):
            if out['marg'][i]:
                continue
            hits = 0
            for l in range(1, 8):
                Tl = T[i, l].reshape(3, 4)
                lv = panda['link_verts'][panda['link_vert_off'][l]:panda['link_vert_off'][l + 1]].astype(np.float64)
                lw = lv @ Tl[:, :3].T + Tl[:, 3]
                if kind == O.ROBOT_TO_OBS:
                    le = panda['link_edges'][panda['link_edge_off'][l]:panda['link_edge_off'][l + 1]]
                    P, Q = lw[le[:, 0]][:, None], lw[le[:, 1]][:, None]
                    h = _seg_tri_numpy(P, Q, tri[None, :, 0], tri[None, :, 1], tri[None, :, 2])
                    hits += int(h.any(axis=1).sum())
                else:
                    lt = panda['link_tris'][panda['link_tri_off'][l]:panda['link_tri_off'][l + 1]]
                    lt3 = lw[lt]
                    h = _seg_tri_numpy(sedge[:, None, 0], sedge[:, None, 1], lt3[None, :, 0], lt3[None, :, 1],
                                       lt3[None, :, 2])
                    hits += int(h.sum())
            assert out['count'][i] == hits, (kind, i)
            assert out['hit'][i] == (hits > 0)
            checked += 1
    assert checked >= 20


def test_sweep_oracle_linear_brute_force(panda):
    mesh = scenes.random_scene(1, 2, 0, seed=8)
    sph = scenes.synth_spheres(panda, per_link=2, seed=0)
    q, off = scenes.random_walk_trajectories(panda, 6, 5, seed=1)
    R, S = O.Robot(panda, spheres=sph), O.Scene(mesh)
    out = O.sweep(False, R, S, q, off)
    T = O.fk(panda, q)
    sv = mesh.verts.astype(np.float64)
    for t in range(6):
        for g in range(4):
            hit = False
            for s in range(len(sph[1])):
                l = sph[2][s]
                c0 = T[off[t] + g, l].reshape(3, 4) @ np.append(sph[0][s], 1.0)
                c1 = T[off[t] + g + 1, l].reshape(3, 4) @ np.append(sph[0][s], 1.0)
                if any(O.seg_seg(sv[e[0]], sv[e[1]], c0, c1) <= sph[1][s] for e in S.edges):
                    hit = True
            assert out['seg_hit'][out['seg_off'][t] + g] == hit


def test_sweep_quad_oracle_segments_and_endpoints(panda):
    sph = scenes.synth_spheres(panda, per_link=2, seed=0)
    q, off = scenes.random_walk_trajectories(panda, 4, [8, 9, 16, 3], seed=2)
    R, S = O.Robot(panda, spheres=sph), O.Scene(scenes.discrete_small())
    a = O.sweep(True, R, S, q, off)
    b = O.sweep(True, R, S, q, off, endpoints=False)
    assert a['seg_off'][-1] == b['seg_off'][-1] + 8
    # dropping the end spheres can only remove hits
    assert np.all(b['traj_hit'] <= a['traj_hit'])


def _winding(p, tri):
    """Generalised winding number of a closed triangle mesh at p (solid angles,
    Van Oosterom & Strackee): about 1 inside, 0 outside - independent of ray
    parity."""
    a, b, c = tri[:, 0] - p, tri[:, 1] - p, tri[:, 2] - p
    la, lb, lc = (np.linalg.norm(x, axis=1) for x in (a, b, c))
    num = np.einsum('ij,ij->i', a, np.cross(b, c))
    den = la * lb * lc + np.einsum('ij,ij->i', a, b) * lc + np.einsum('ij,ij->i', b, c) * la + \
        np.einsum('ij,ij->i', c, a) * lb
    return float(2.0 * np.arctan2(num, den).sum() / (4 * np.pi))


def test_containment_oracle_against_winding_numbers(panda):
    """A 1 mm box whose first vertex is a link's vertex-mean point (or a point
    pushed out from it): the oracle's
    ray-parity containment equals the winding-number truth (inside some
    checked link), for every pose without a surface crossing."""
    q = scenes.uniform_poses(panda, 40, seed=5)
    T = O.fk(panda, q)
    R = O.Robot(panda)
    checked = inside_seen = 0
    for i in range(len(q)):
        l = 1 + i % 7
        lv = panda['link_verts'][panda['link_vert_off'][l]:panda['link_vert_off'][l + 1]].astype(np.float64)
        Tl = T[i, l].reshape(3, 4)
        P = lv.mean(axis=0) @ Tl[:, :3].T + Tl[:, 3]
        if i % 2:  # half the points pushed out to 3-12 cm from the link's centre
            d = np.random.default_rng(i).normal(size=3)
            P = P + (0.03 + 0.09 * (i % 4) / 3) * d / np.linalg.norm(d)
        v, t = scenes.box_mesh(P + 0.0005, [0.001] * 3)
        mesh = scenes.Mesh(v, t, [0, 12])
        assert np.allclose(mesh.verts[0], P, atol=1e-6)
        S = O.Scene(mesh)
        hit = O.discrete(O.ROBOT_TO_OBS, R, S, q[i:i + 1])['hit'] | O.discrete(O.OBS_TO_ROBOT, R, S, q[i:i + 1])['hit']
        if hit[0]:
            continue
        w = []
        P32 = mesh.verts[0].astype(np.float64)
        for k in range(1, 8):
            Tk = T[i, k].reshape(3, 4)
            kv = panda['link_verts'][panda['link_vert_off'][k]:panda['link_vert_off'][k + 1]].astype(np.float64)
            kt = panda['link_tris'][panda['link_tri_off'][k]:panda['link_tri_off'][k + 1]]
            w.append(_winding(P32, (kv @ Tk[:, :3].T + Tk[:, 3])[kt]))
        w = np.abs(np.array(w))
        if np.any(np.abs(w - 0.5) < 0.2):
            continue  # too close to a surface for either method to be sharp
        out = O.containment(R, S, q[i:i + 1])
        if out['band'][0]:
            continue
        assert out['contain'][0] == int(np.any(w > 0.5)), (i, w)
        checked += 1
        inside_seen += int(out['contain'][0])
    assert checked >= 20 and 0 < inside_seen < checked


def test_containment_oracle_enclosing_box(panda):
    """The robot inside one large box: no surface crossing, every pose contained;
    far away: nothing."""
    q = scenes.uniform_poses(panda, 16, seed=6)
    R = O.Robot(panda)
    v, t = scenes.box_mesh([0, 0, 0.5], [6, 6, 6])
    S = O.Scene(scenes.Mesh(v, t, [0, 12]))
    assert O.discrete(O.ROBOT_TO_OBS, R, S, q)['hit'].sum() == 0
    out = O.containment(R, S, q)
    assert out['contain'].all() and not out['band'].any()
    v, t = scenes.box_mesh([20, 0, 0], [1, 1, 1])
    S = O.Scene(scenes.Mesh(v, t, [0, 12]))
    assert O.containment(R, S, q)['contain'].sum() == 0
    assert O.containment(R, S, q, skip=np.ones(16))['contain'].sum() == 0
