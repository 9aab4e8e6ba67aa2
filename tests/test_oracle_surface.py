"""The oracle's restatement of the reference's sweep semantics (no GPU):
directed loop edges (RTCD/Meshes/mesh.h:378-620) and the entering-ray
predicate of the curve intersectors (a directed edge hits a primitive when it
starts outside the primitive's closed solid and reaches it; round caps on the
linear capsules, flat caps on the quadratic pieces)."""
import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import scenes


def test_loop_edges_tetrahedron_known_answer():
    """Worked by hand through the upstream rules: T0 all forward (no edge
    decided); T1 one backward edge -> the other two backward; T2 one forward,
    one backward -> the forward one doubled, the open edge backward; T3 two
    forward, one backward -> the backward one doubled."""
    tet = np.array([[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]], np.uint32)
    got = O.loop_edges(tet).tolist()
    assert got == [[0, 1], [1, 2], [2, 0], [0, 2], [3, 0], [3, 1], [1, 3], [2, 3]]


def _is_loop(tri, dset):
    f = sum((int(tri[i]), int(tri[(i + 1) % 3])) in dset for i in range(3))
    b = sum((int(tri[(i + 1) % 3]), int(tri[i])) in dset for i in range(3))
    return f == 3 or b == 3


@pytest.mark.parametrize('which', ['box', 'ico2', 'small', 'sweep'])
def test_loop_edges_close_every_triangle(which):
    if which == 'box':
        v, t = scenes.box_mesh([0, 0, 0], [1, 2, 3])
    elif which == 'ico2':
        v, t = scenes.icosphere(2)
    else:
        m = scenes.discrete_small() if which == 'small' else scenes.sweep_scene()
        t = m.tris
    le = O.loop_edges(t)
    d = set(map(tuple, le.tolist()))
    assert len(d) == len(le)  # each directed edge once
    assert all(_is_loop(tri, d) for tri in t)
    und = {tuple(sorted(e)) for e in O.unique_edges(t).tolist()}
    assert {tuple(sorted(e)) for e in d} == und  # every mesh edge, in at least one direction
    assert len(und) <= len(le) <= 2 * len(und)


def _cap(quad, p, q, r=0.1):
    if quad:
        return O.surface_pair(1, p, q, [0, 0, 0], [0.5, 0, 0], [1, 0, 0], r)
    return O.surface_pair(0, p, q, [0, 0, 0], [1, 0, 0], [1, 0, 0], r)


@pytest.mark.parametrize('quad,p,q,hit,band', [
    (0, [0.5, 0.5, 0], [0.5, -0.5, 0], True, False),     # crosses the capsule
    (0, [0.5, 0.0, 0], [0.5, 0.5, 0], False, False),     # starts on the axis: leaves, never enters
    (0, [0.5, 0.05, 0], [0.5, 0.08, 0], False, False),   # wholly inside (a solid hit)
    (0, [0.5, 0.1, -1], [0.5, 0.1, 1], True, True),      # tangent: distance exactly r
    (0, [-0.05, 0.5, 0], [-0.05, -0.5, 0], True, False), # through the round start cap
    (1, [-0.05, 0.5, 0], [-0.05, -0.5, 0], False, False),  # beyond the flat start cap
    (1, [0.5, 0.5, 0], [0.5, -0.5, 0], True, False),
    (1, [-0.5, 0.05, 0], [0.5, 0.05, 0], True, False),   # enters through the cap disk (closed caps)
    (1, [0.5, 0.05, 0], [1.5, 0.05, 0], False, False),   # starts inside, leaves through the end cap
    (1, [1.05, 0, 0.5], [1.05, 0, -0.5], False, False),  # beyond the flat end cap
    (1, [0.0, 0.5, 0], [0.0, -0.5, 0], True, True),      # in the start cap's plane
])
def test_surface_pair_known_answers(quad, p, q, hit, band):
    assert _cap(quad, p, q) == (hit, band)


def test_surface_pair_curved_piece_against_sampling():
    """A curved piece: the entering-ray decision equals a dense sampling of
    the segment against the sphere-swept, plane-cut solid (pairs whose
    decision flips within 1 mm of the sampled boundary are skipped)."""
    rng = np.random.default_rng(3)
    B0, B1, B2 = np.array([0.0, 0, 0]), np.array([0.3, 0.25, 0]), np.array([0.6, 0, 0.05])
    r = 0.05
    n0 = (B1 - B0) / np.linalg.norm(B1 - B0)
    n1 = (B2 - B1) / np.linalg.norm(B2 - B1)
    u = np.linspace(0, 1, 1001)
    C = ((1 - u) ** 2)[:, None] * B0 + (2 * u * (1 - u))[:, None] * B1 + (u ** 2)[:, None] * B2

    def margin(x):  # > 0 inside the solid, < 0 outside (approximate signed clearance)
        d = np.min(np.linalg.norm(C[None] - x[:, None], axis=2), axis=1)
        s0 = (x - B0) @ n0
        s1 = (B2 - x) @ n1
        return np.minimum(np.minimum(r - d, s0), s1)

    checked = hits = 0
    for _ in range(500):
        uu = rng.uniform(-0.1, 1.1)
        aim = (1 - uu) ** 2 * B0 + 2 * uu * (1 - uu) * B1 + uu ** 2 * B2 + rng.normal(size=3) * 0.04
        d = rng.normal(size=3)
        p = aim + d / np.linalg.norm(d) * rng.uniform(0.0, 0.15)
        q = aim + (aim - p) * rng.uniform(-0.5, 1.0)
        t = np.linspace(0, 1, 401)
        x = p[None] + t[:, None] * (q - p)[None]
        m = margin(x)
        dl = 1e-3  # beyond the sampling error of the margin
        if m[0] < -dl and np.any(m > dl):
            want = True
        elif m[0] > dl or np.all(m < -dl):
            want = False
        else:
            continue
        got, band = O.surface_pair(1, p, q, B0, B1, B2, r)
        assert not band
        assert got == want, (p, q)
        checked += 1
        hits += int(want)
    assert checked > 200 and 20 < hits < checked - 20


def test_surface_sweeps_are_subsets_of_solid(panda):
    """Per segment, a surface hit is a solid hit (the flat-capped piece lies in
    the round-capped one and every loop edge is a mesh edge); the reverse fails
    where an edge lies wholly inside a capsule."""
    sph = scenes.synth_spheres(panda, per_link=2, seed=0)
    R, S = O.Robot(panda, spheres=sph), O.Scene(scenes.discrete_small())
    for quad in (False, True):
        q, off = scenes.random_walk_trajectories(panda, 24, [9] * 24, seed=4)
        a = O.sweep(quad, R, S, q, off, endpoints=False)
        b = O.sweep(quad, R, S, q, off, surface=True)
        assert np.array_equal(a['seg_off'], b['seg_off'])
        ok = (a['seg_band'] == 0) & (b['seg_band'] == 0)
        assert np.all(b['seg_hit'][ok] <= a['seg_hit'][ok])
        assert a['seg_hit'].sum() > 0


def test_surface_sweep_linear_brute_force(panda):
    """The BVH-accelerated surface sweep equals every (loop edge, capsule) pair
    evaluated one by one."""
    mesh = scenes.random_scene(1, 2, 0, seed=8)
    sph = scenes.synth_spheres(panda, per_link=2, seed=0)
    q, off = scenes.random_walk_trajectories(panda, 6, 5, seed=1)
    R, S = O.Robot(panda, spheres=sph), O.Scene(mesh)
    out = O.sweep(False, R, S, q, off, surface=True)
    S.loop()
    T = O.fk(panda, q)
    sv = mesh.verts.astype(np.float64)
    for t in range(6):
        for g in range(4):
            hit = False
            for s in range(len(sph[1])):
                l = sph[2][s]
                c0 = T[off[t] + g, l].reshape(3, 4) @ np.append(sph[0][s], 1.0)
                c1 = T[off[t] + g + 1, l].reshape(3, 4) @ np.append(sph[0][s], 1.0)
                for e in S.loop_edges:
                    if O.surface_pair(0, sv[e[0]], sv[e[1]], c0, c1, c1, sph[1][s])[0]:
                        hit = True
                        break
            assert out['seg_hit'][out['seg_off'][t] + g] == hit


@pytest.mark.parametrize('which', ['tet', 'small', 'sweep', 'shelf'])
def test_library_loop_edges_equal_oracle(which):
    """The library's own loop-edge builder (host code, rtcd_loop_edges) and
    the oracle's restatement agree edge for edge, in order."""
    from rtcollisiondetection_b200 import rtcd
    if which == 'tet':
        t = np.array([[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]], np.uint32)
    elif which == 'small':
        t = scenes.discrete_small().tris
    elif which == 'sweep':
        t = scenes.sweep_scene().tris
    else:
        t = scenes.reference_scene('simple').tris
    assert np.array_equal(rtcd.loop_edges(t), O.loop_edges(t))
