"""Seeded synthetic inputs: robot model, obstacle scenes, poses and trajectories.

Every generator is deterministic for a given seed (numpy PCG64).  The shapes,
sizes and value ranges follow the benchmark workloads of the detector:

* ``discrete_small``  - 12 axis-aligned boxes (extents U(0.02, 0.6) m) and 16
  level-2 icospheres (radius U(0.03, 0.1) m) in the 1 m cube in front of the
  robot, x in [0, 1], y in [-0.5, 0.5], z in [0, 1] (5,264 triangles);
* ``discrete_dense``  - 64 boxes (extents U(0.02, 0.4) m), 256 level-3
  icospheres (radius U(0.03, 0.1) m) and one 100,000-triangle sphere
  (radius 0.15 m) with seeded radial displacement noise of amplitude 0.1 r,
  about 428k triangles (``ico_level=2`` gives the 183k variant), spread over
  the robot-centred box x, y in [-1.5, 1.5], z in [0, 1.5]: packed into the
  1 m cube every random pose collides;
* ``sweep_scene``     - 12 boxes (extents U(0.02, 0.3) m) and 155 level-2
  icospheres (radius U(0.02, 0.06) m), 49,744 triangles, over the same
  robot-centred box.

Poses are uniform within the joint limits; trajectories are random walks with
N(0, 0.1) rad steps clipped to the limits.  The robot model (Panda) comes from
``data/panda.npz``.
"""
import os
import numpy as np

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data')
WORKSPACE_LO = np.array([0.0, -0.5, 0.0])
WORKSPACE_HI = np.array([1.0, 0.5, 1.0])
WIDE_LO = np.array([-1.5, -1.5, 0.0])
WIDE_HI = np.array([1.5, 1.5, 1.5])


class Mesh:
    """Triangle soup with per-obstacle triangle ranges."""

    def __init__(self, verts, tris, obstacle_tri_off):
        self.verts = np.ascontiguousarray(verts, dtype=np.float32)
        self.tris = np.ascontiguousarray(tris, dtype=np.uint32)
        self.obstacle_tri_off = np.ascontiguousarray(obstacle_tri_off, dtype=np.uint32)

    @property
    def n_tris(self):
        return len(self.tris)

    @property
    def n_obstacles(self):
        return len(self.obstacle_tri_off) - 1


def load_panda():
    """The Panda model arrays (see ``data/make_panda.py``)."""
    d = np.load(os.path.join(DATA_DIR, 'panda.npz'))
    return {k: d[k] for k in d.files}


def synth_spheres(robot, per_link=8, seed=0):
    """``per_link`` spheres per link: centres are seeded random vertices of that
    link mesh, radii U(0.02, 0.08) m."""
    rng = np.random.default_rng(seed)
    vo = robot['link_vert_off']
    centers, radii, links = [], [], []
    for l in range(len(vo) - 1):
        idx = rng.choice(int(vo[l + 1] - vo[l]), size=per_link, replace=False)
        centers.append(robot['link_verts'][vo[l] + idx])
        radii.append(rng.uniform(0.02, 0.08, size=per_link))
        links += [l] * per_link
    return (np.concatenate(centers).astype(np.float32), np.concatenate(radii).astype(np.float32),
            np.asarray(links, np.uint32))


# --------------------------------------------------------------------------- shapes
def box_mesh(center, extent):
    h = 0.5 * np.asarray(extent, np.float64)
    c = np.asarray(center, np.float64)
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64) * h + c
    # outward-facing triangles of the 6 faces
    t = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                  [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.uint32)
    return v, t


def icosphere(level):
    p = (1.0 + 5 ** 0.5) / 2
    v = [[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
         [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]]
    v = [np.array(x, np.float64) / np.linalg.norm(x) for x in v]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
         [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    for _ in range(level):
        cache, nf = {}, []

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[k] = len(v) - 1
            return cache[k]
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = nf
    return np.array(v, np.float64), np.array(f, np.uint32)


def latlong_sphere(n_lon, n_lat):
    """Closed UV sphere: poles + (n_lat - 1) rings of n_lon vertices;
    2 * n_lon * (n_lat - 1) triangles."""
    verts = [[0.0, 0.0, 1.0]]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            verts.append([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    verts.append([0.0, 0.0, -1.0])
    tris = []
    ring = lambda i, j: 1 + (i - 1) * n_lon + (j % n_lon)
    for j in range(n_lon):
        tris.append([0, ring(1, j), ring(1, j + 1)])
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            tris += [[a, c, d], [a, d, b]]
    south = len(verts) - 1
    for j in range(n_lon):
        tris.append([south, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)])
    return np.array(verts, np.float64), np.array(tris, np.uint32)


def _assemble(parts):
    verts, tris, off = [], [], [0]
    nv = 0
    for v, t in parts:
        verts.append(v)
        tris.append(t + nv)
        nv += len(v)
        off.append(off[-1] + len(t))
    return Mesh(np.concatenate(verts), np.concatenate(tris), np.asarray(off, np.uint32))


def random_scene(n_boxes, n_icos, ico_level, seed=0, big_sphere_tris=0, big_sphere_radius=0.15,
                 ico_r=(0.03, 0.1), box_ext=(0.02, 0.6), workspace=(WORKSPACE_LO, WORKSPACE_HI)):
    rng = np.random.default_rng(seed)
    lo, hi = workspace
    parts = []
    for _ in range(n_boxes):
        parts.append(box_mesh(rng.uniform(lo, hi), rng.uniform(box_ext[0], box_ext[1], size=3)))
    uv, ut = icosphere(ico_level)
    for _ in range(n_icos):
        r = rng.uniform(*ico_r)
        parts.append((uv * r + rng.uniform(lo, hi), ut))
    if big_sphere_tris:
        n_lon = 250
        n_lat = big_sphere_tris // (2 * n_lon) + 1
        sv, st = latlong_sphere(n_lon, n_lat)
        radial = big_sphere_radius * (1.0 + 0.1 * rng.uniform(-1.0, 1.0, size=len(sv)))
        parts.append((sv * radial[:, None] + rng.uniform(lo, hi), st))
    return _assemble(parts)


def discrete_small(seed=0):
    """12 boxes + 16 level-2 icospheres in the 1 m cube: 5,264 triangles."""
    return random_scene(12, 16, 2, seed)


def discrete_dense(seed=0, ico_level=3):
    """64 boxes + 256 icospheres + the 100k noisy sphere (level 3: ~428k triangles)."""
    return random_scene(64, 256, ico_level, seed, big_sphere_tris=100_000, box_ext=(0.02, 0.4),
                        workspace=(WIDE_LO, WIDE_HI))


def discrete_dense_cube(seed=0):
    """The dense composition packed into the 1 m workspace cube of the small
    scene, as the configuration literally reads (box extents U(0.02, 0.6) m):
    428,448 triangles in front of the robot, where nearly every pose collides."""
    return random_scene(64, 256, 3, seed, big_sphere_tris=100_000)


def sweep_scene(seed=0):
    """12 boxes + 155 level-2 icospheres: 49,744 triangles."""
    return random_scene(12, 155, 2, seed, ico_r=(0.02, 0.06), box_ext=(0.02, 0.3), workspace=(WIDE_LO, WIDE_HI))


def sweep_scene_sparse(seed=0):
    """12 boxes + 38 level-3 icospheres over the same box (48,784 triangles):
    fewer, finer obstacles, so about 40 % of the 32-waypoint random walks
    collide instead of nearly all."""
    return random_scene(12, 38, 3, seed, ico_r=(0.02, 0.06), box_ext=(0.02, 0.3), workspace=(WIDE_LO, WIDE_HI))


def served_large_scene(seed=0):
    """Dense scene plus 225 extra level-2 icospheres (~500k triangles)."""
    base = discrete_dense(seed)
    extra = random_scene(0, 225, 2, seed + 1, workspace=(WIDE_LO, WIDE_HI))
    v = np.concatenate([base.verts, extra.verts])
    t = np.concatenate([base.tris, extra.tris + len(base.verts)])
    off = np.concatenate([base.obstacle_tri_off, extra.obstacle_tri_off[1:] + base.obstacle_tri_off[-1]])
    return Mesh(v, t, off)


def reference_scene(name):
    """The reference's benchmark shelves ('simple', 'medium', 'dense': 15,008 /
    71,746 / 202,330 triangles), one obstacle per placed model, from
    ``data/ref_scenes.npz`` (see ``data/make_ref_scenes.py``)."""
    d = np.load(os.path.join(DATA_DIR, 'ref_scenes.npz'))
    verts, tris, off, nv = [], [], [0], 0
    for m, t in zip(d['scene_%s_models' % name], d['scene_%s_offsets' % name]):
        v = d['model_%s_verts' % m] + t.astype(np.float32)   # identity pose translated, in float
        verts.append(v)
        tris.append(d['model_%s_tris' % m] + np.uint32(nv))
        nv += len(v)
        off.append(off[-1] + len(d['model_%s_tris' % m]))
    return Mesh(np.concatenate(verts), np.concatenate(tris), off)


# --------------------------------------------------------------------------- queries
def uniform_poses(robot, n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(robot['lower'], robot['upper'], size=(n, len(robot['lower']))).astype(np.float32)


def random_walk_trajectories(robot, n_traj, n_wp, seed=0, step=0.1):
    """Random-walk trajectories.  ``n_wp`` is an int (all equal) or an array of
    per-trajectory waypoint counts.  Returns (q[total_wp, dof], traj_off[n+1])."""
    rng = np.random.default_rng(seed)
    lo, hi = robot['lower'].astype(np.float64), robot['upper'].astype(np.float64)
    counts = np.full(n_traj, n_wp, np.int64) if np.isscalar(n_wp) else np.asarray(n_wp, np.int64)
    off = np.zeros(n_traj + 1, np.uint32)
    off[1:] = np.cumsum(counts)
    q = np.empty((int(off[-1]), len(lo)), np.float64)
    for i in range(n_traj):
        x = rng.uniform(lo, hi)
        for k in range(counts[i]):
            if k:
                x = np.clip(x + rng.normal(0.0, step, size=len(lo)), lo, hi)
            q[off[i] + k] = x
    return q.astype(np.float32), off


def log_uniform_counts(n, lo, hi, seed=0):
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=n))).astype(np.int64)


def quad_ctrl_count(n_wp):
    """Control points of the quadratic fit for a trajectory of ``n_wp`` waypoints."""
    return max(3, -(-int(n_wp) // 2))
