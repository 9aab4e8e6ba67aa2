"""ctypes binding of the FP64 oracle (``oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product package never imports it.
"""
import ctypes as C
import os
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liboracle.so')
OBS_TO_ROBOT, ROBOT_TO_OBS = 0, 1


def build():
    subprocess.check_call(['make', '-s', '-C', HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, 'oracle.c')):
            build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


F, U, D, B = C.c_float, C.c_uint, C.c_double, C.c_ubyte


class OrcRobot(C.Structure):
    _fields_ = [('dof', C.c_int), ('cos_mask', C.POINTER(F)), ('sin_mask', C.POINTER(F)), ('one_mask', C.POINTER(F)),
                ('base_tf', C.POINTER(F)), ('n_links', C.c_int), ('link_verts', C.POINTER(F)),
                ('link_vert_off', C.POINTER(U)), ('link_tris', C.POINTER(U)), ('link_tri_off', C.POINTER(U)),
                ('link_edges', C.POINTER(U)), ('link_edge_off', C.POINTER(U)), ('skip_base', C.c_int),
                ('n_spheres', C.c_int), ('sphere_centers', C.POINTER(F)), ('sphere_radii', C.POINTER(F)),
                ('sphere_links', C.POINTER(U))]


class OrcScene(C.Structure):
    _fields_ = [('n_verts', C.c_int), ('verts', C.POINTER(F)), ('n_tris', C.c_int), ('tris', C.POINTER(U)),
                ('n_edges', C.c_int), ('edges', C.POINTER(U))]


class OrcWork(C.Structure):
    _fields_ = [('node_tests', C.c_uint64), ('prim_tests', C.c_uint64)]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class Robot:
    """Holds the arrays alive for the C struct."""

    def __init__(self, model, spheres=None, skip_base=True):
        self.a = {
            'cos': _c(model['cos_mask'], np.float32), 'sin': _c(model['sin_mask'], np.float32),
            'one': _c(model['one_mask'], np.float32), 'base': _c(model['base_tf'], np.float32),
            'lv': _c(model['link_verts'], np.float32), 'lvo': _c(model['link_vert_off'], np.uint32),
            'lt': _c(model['link_tris'], np.uint32), 'lto': _c(model['link_tri_off'], np.uint32),
            'le': _c(model['link_edges'], np.uint32), 'leo': _c(model['link_edge_off'], np.uint32),
        }
        if spheres is None:
            spheres = (model['sphere_centers'], model['sphere_radii'], model['sphere_links'])
        self.a['sc'] = _c(spheres[0], np.float32)
        self.a['sr'] = _c(spheres[1], np.float32)
        self.a['sl'] = _c(spheres[2], np.uint32)
        a = self.a
        self.dof = a['cos'].shape[0]
        self.s = OrcRobot(self.dof, _p(a['cos'], F), _p(a['sin'], F), _p(a['one'], F), _p(a['base'], F),
                          len(a['lvo']) - 1, _p(a['lv'], F), _p(a['lvo'], U), _p(a['lt'], U), _p(a['lto'], U),
                          _p(a['le'], U), _p(a['leo'], U), int(bool(skip_base)), len(a['sr']), _p(a['sc'], F),
                          _p(a['sr'], F), _p(a['sl'], U))


def unique_edges(tris):
    tris = _c(tris, np.uint32)
    out = np.empty((max(1, 3 * len(tris)), 2), np.uint32)
    n = lib().orc_unique_edges(_p(tris, U), C.c_int(len(tris)), _p(out, U))
    return out[:n].copy()


def loop_edges(tris):
    """Directed loop edges of a watertight mesh (upstream RTCD/Meshes/mesh.h:378-620), (m, 2) uint32."""
    tris = _c(tris, np.uint32)
    out = np.empty((max(1, 6 * len(tris)), 2), np.uint32)
    n = lib().orc_loop_edges(_p(tris, U), C.c_int(len(tris)), _p(out, U))
    if n < 0:
        raise ValueError('mesh is not watertight: a triangle does not close a loop')
    return out[:n].copy()


class Scene:
    def __init__(self, mesh):
        self.verts = _c(mesh.verts, np.float32)
        self.tris = _c(mesh.tris, np.uint32)
        off = getattr(mesh, 'obstacle_tri_off', None)
        self.obstacle_tri_off = _c(off if off is not None else [0, len(self.tris)], np.uint32)
        self.edges = unique_edges(self.tris)
        self.s = OrcScene(len(self.verts), _p(self.verts, F), len(self.tris), _p(self.tris, U), len(self.edges),
                          _p(self.edges, U))
        self._loop = None

    def loop(self):
        """The scene with its directed loop edges in place of the unique edges (surface semantics)."""
        if self._loop is None:
            self.loop_edges = loop_edges(self.tris)
            self._loop = OrcScene(len(self.verts), _p(self.verts, F), len(self.tris), _p(self.tris, U),
                                  len(self.loop_edges), _p(self.loop_edges, U))
        return self._loop


def fk(model, q):
    q = _c(q, np.float32)
    n, dof = q.shape
    T = np.empty((n, dof + 1, 12), np.float64)
    lib().orc_fk(C.c_int(dof), _p(_c(model['cos_mask'], np.float32), F), _p(_c(model['sin_mask'], np.float32), F),
                 _p(_c(model['one_mask'], np.float32), F), _p(_c(model['base_tf'], np.float32), F), _p(q, F),
                 C.c_int(n), _p(T, D))
    return T


def lbvh(plo, phi):
    """Canonical LBVH: (codes, perm, child[n-1,2], node_lo[n-1,3], node_hi[n-1,3])."""
    plo, phi = _c(plo, np.float32), _c(phi, np.float32)
    n = len(plo)
    codes = np.empty(n, np.uint32)
    perm = np.empty(n, np.uint32)
    m = max(n - 1, 1)
    child = np.empty((m, 2), np.int32)
    nlo = np.empty((m, 3), np.float32)
    nhi = np.empty((m, 3), np.float32)
    lib().orc_lbvh_build(_p(plo, F), _p(phi, F), C.c_int(n), _p(codes, U), _p(perm, U), _p(child, C.c_int),
                         _p(nlo, F), _p(nhi, F))
    return codes, perm, child[:n - 1], nlo[:n - 1], nhi[:n - 1]


def threads_default():
    return os.cpu_count() or 1


def discrete(kind, robot, scene, q, eps=1e-5, threads=None, work=False):
    """Returns dict(hit, count, band[, node_tests, prim_tests]) per pose."""
    q = _c(q, np.float32)
    n = len(q)
    hit = np.zeros(n, np.uint8)
    band = np.zeros(n, np.uint8)
    marg = np.zeros(n, np.uint8)
    count = np.zeros(n, np.uint32)
    w = (OrcWork * n)() if work else None
    lib().orc_discrete(C.c_int(kind), C.byref(robot.s), C.byref(scene.s), _p(q, F), C.c_int(n), D(eps),
                       C.c_int(threads or threads_default()), _p(hit, B), _p(count, U), _p(band, B), _p(marg, B), w)
    out = {'hit': hit, 'count': count, 'band': band, 'marg': marg}
    if work:
        arr = np.ctypeslib.as_array(w)
        out['node_tests'] = arr['node_tests'].copy()
        out['prim_tests'] = arr['prim_tests'].copy()
    return out


def containment(robot, scene, q, skip=None, eps=1e-5, threads=None):
    """Containment of poses without a surface crossing (skip[pose] != 0 skips
    a pose): dict(contain, band) - a link vertex inside an obstacle or an
    obstacle vertex inside a link, by ray parity (no upstream counterpart)."""
    q = _c(q, np.float32)
    n = len(q)
    contain = np.zeros(n, np.uint8)
    band = np.zeros(n, np.uint8)
    sk = None if skip is None else _c(np.asarray(skip) != 0, np.uint8)
    off = scene.obstacle_tri_off
    lib().orc_containment(C.byref(robot.s), C.byref(scene.s), _p(off, U), C.c_int(len(off) - 1), _p(q, F), C.c_int(n),
                          D(eps), C.c_int(threads or threads_default()), _p(sk, B), _p(contain, B), _p(band, B))
    return {'contain': contain, 'band': band}


class PreparedDiscrete:
    """Acceleration structures built once; ``run`` times the queries alone."""

    def __init__(self, kind, robot, scene):
        self.robot, self.scene = robot, scene
        lib().orc_discrete_prepare.restype = C.c_void_p
        self.h = C.c_void_p(lib().orc_discrete_prepare(C.c_int(kind), C.byref(robot.s), C.byref(scene.s)))

    def flags(self, q, threads=None):
        """Flags only, each pose stopping at its first hit."""
        q = _c(q, np.float32)
        hit = np.zeros(len(q), np.uint8)
        lib().orc_discrete_run(self.h, _p(q, F), C.c_int(len(q)), D(1e-5), C.c_int(threads or threads_default()),
                               C.c_int(1), _p(hit, B), None, None, None, None)
        return hit

    def close(self):
        if self.h:
            lib().orc_discrete_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def quad_ctrl_count(n_wp):
    return max(3, -(-int(n_wp) // 2))


def sweep_seg_offsets(traj_off, quad, endpoints=True):
    counts = np.diff(np.asarray(traj_off, np.int64))
    if quad:
        segs = np.array([quad_ctrl_count(c) - 2 + (2 if endpoints else 0) for c in counts], np.int64)
    else:
        segs = np.maximum(counts - 1, 0)
    off = np.zeros(len(counts) + 1, np.uint32)
    off[1:] = np.cumsum(segs)
    return off


def sweep(quad, robot, scene, q, traj_off, eps=1e-5, threads=None, endpoints=True, work=False, surface=False):
    """Returns dict(traj_hit, traj_band, seg_hit, seg_band, seg_off[, node_tests, prim_tests]).

    surface=False: solid semantics over the unique edges; surface=True: the
    reference's entering-ray semantics over the directed loop edges, no end
    spheres (endpoints is ignored)."""
    q = _c(q, np.float32)
    traj_off = _c(traj_off, np.uint32)
    nt = len(traj_off) - 1
    if surface:
        endpoints = False
    seg_off = sweep_seg_offsets(traj_off, quad, endpoints)
    th = np.zeros(nt, np.uint8)
    tb = np.zeros(nt, np.uint8)
    tm = np.zeros(nt, np.uint8)
    tc = np.zeros(nt, np.uint32)
    sh = np.zeros(max(1, int(seg_off[-1])), np.uint8)
    sb = np.zeros(max(1, int(seg_off[-1])), np.uint8)
    w = (OrcWork * nt)() if work else None
    sc = scene.loop() if surface else scene.s
    lib().orc_sweep(C.c_int(int(quad)), C.c_int(int(endpoints)), C.c_int(int(surface)), C.byref(robot.s), C.byref(sc),
                    _p(q, F),
                    _p(traj_off, U), C.c_int(nt), D(eps), C.c_int(threads or threads_default()), _p(th, B), _p(tb, B),
                    _p(tm, B), _p(tc, U), _p(seg_off, U), _p(sh, B), _p(sb, B), w)
    out = {'traj_hit': th, 'traj_band': tb, 'traj_marg': tm, 'traj_count': tc, 'seg_hit': sh[:seg_off[-1]],
           'seg_band': sb[:seg_off[-1]], 'seg_off': seg_off}
    if work:
        arr = np.ctypeslib.as_array(w)
        out['node_tests'] = arr['node_tests'].copy()
        out['prim_tests'] = arr['prim_tests'].copy()
    return out


def fit_weights(nc, nt):
    W = np.empty((nc, nt), np.float64)
    rc = lib().orc_fit_weights(C.c_int(nc), C.c_int(nt), _p(W, D))
    if rc:
        raise ValueError('bad fit size %d x %d' % (nc, nt))
    return W


def seg_tri(p, q, a, b, c):
    arr = [_c(x, np.float64) for x in (p, q, a, b, c)]
    m = C.c_double()
    h = lib().orc_seg_tri(*[_p(x, D) for x in arr], C.byref(m))
    return bool(h), m.value


def seg_seg(p1, q1, p2, q2):
    lib().orc_seg_seg.restype = C.c_double
    arr = [_c(x, np.float64) for x in (p1, q1, p2, q2)]
    return lib().orc_seg_seg(*[_p(x, D) for x in arr])


def seg_quad(p, q, b0, b1, b2):
    lib().orc_seg_quad.restype = C.c_double
    arr = [_c(x, np.float64) for x in (p, q, b0, b1, b2)]
    return lib().orc_seg_quad(*[_p(x, D) for x in arr])


def surface_pair(quad, p, q, b0, b1, b2, r, eps=1e-5):
    """One (directed edge p -> q, primitive) pair under the reference's
    entering-ray semantics: (hit, band)."""
    arr = [_c(x, np.float64) for x in (p, q, b0, b1, b2)]
    hit, band = C.c_int(), C.c_int()
    lib().orc_surface_pair(C.c_int(int(quad)), *[_p(x, D) for x in arr], D(r), D(eps), C.byref(hit), C.byref(band))
    return bool(hit.value), bool(band.value)
