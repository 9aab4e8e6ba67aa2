"""ctypes binding of ``librtcd_b200.so`` (include/rtcd.h) and a Python mirror
of the upstream detector interface.

The upstream API is ``RTCD::CollisionDetector<NSTREAM, LinkType>``
(RTCD/CollisionDetector/CollisionDetector.h:18-157) driven as
``setupScene -> setupOptix -> setupRobot -> buildSBT`` then per query
``robot->prepareUpdateData(poses, n); setNCheck(n); check(); downloadResult(v)``.
:class:`CollisionDetector` keeps those method names; :class:`Context`,
:class:`Robot`, :class:`Scene` and :class:`Detector` are the thin handle
wrappers.  There is no CPU fallback: a missing library raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'librtcd_b200.so')

OBS_TO_ROBOT, ROBOT_TO_OBS, LINEAR_SWEEP, QUAD_SWEEP = 0, 1, 2, 3
KIND_NAMES = {'ObsToRobot': OBS_TO_ROBOT, 'RobotToObs': ROBOT_TO_OBS, 'Linear': LINEAR_SWEEP, 'Quadratic': QUAD_SWEEP}

CHECK_COUNTS = 1 << 0
CHECK_HOST_BUFFERS = 1 << 1
CHECK_NO_CULL = 1 << 2
CHECK_PLAIN = 1 << 3
CHECK_NO_ENDPOINTS = 1 << 4
CHECK_TIMING = 1 << 5
CHECK_FUSED = 1 << 6
CHECK_GRAPH = 1 << 7
CHECK_CONTAINMENT = 1 << 8
CHECK_TWO_WAY = 1 << 9
CHECK_SURFACE = 1 << 10

STATUS = {0: 'RTCD_OK', 1: 'RTCD_ERR_INVALID_ARGUMENT', 2: 'RTCD_ERR_CUDA', 3: 'RTCD_ERR_OUT_OF_MEMORY',
          4: 'RTCD_ERR_DEVICE_TIMEOUT', 5: 'RTCD_ERR_CAPACITY', 6: 'RTCD_ERR_INTERNAL'}

EXPORTS = ['rtcd_abi_version', 'rtcd_last_error', 'rtcd_context_create', 'rtcd_context_destroy', 'rtcd_robot_create',
           'rtcd_robot_destroy', 'rtcd_scene_create', 'rtcd_scene_destroy', 'rtcd_scene_info', 'rtcd_detector_create',
           'rtcd_detector_destroy', 'rtcd_check', 'rtcd_sync', 'rtcd_segment_offsets', 'rtcd_last_stats',
           'rtcd_robot_fk', 'rtcd_exclusive_scan_u32', 'rtcd_select_flags_u8', 'rtcd_lbvh_build',
           'rtcd_server_create', 'rtcd_server_destroy', 'rtcd_server_submit', 'rtcd_server_wait',
           'rtcd_server_get_stats', 'rtcd_server_reset_stats', 'rtcd_detector_autotune', 'rtcd_server_prepare',
           'rtcd_select_flags_u8_noalloc', 'rtcd_quad_fit_weights', 'rtcd_urdf_chain_parse', 'rtcd_obj_load',
           'rtcd_halton_samples', 'rtcd_knn', 'rtcd_check_edges', 'rtcd_selftest_lookback_timeout',
           'rtcd_loop_edges', 'rtcd_exact_test_probe']


class RTCDError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__('%s: %s' % (STATUS.get(status, status), msg))
        self.status = status


F, U, VP = C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_void_p


class RobotDesc(C.Structure):
    _fields_ = [('dof', C.c_uint32), ('base_tf', F), ('cos_mask', F), ('sin_mask', F), ('one_mask', F),
                ('link_verts', F), ('link_vert_offsets', U), ('link_tris', U), ('link_tri_offsets', U),
                ('link_edges', U), ('link_edge_offsets', U), ('link_obbs', F), ('n_spheres', C.c_uint32),
                ('sphere_centers', F), ('sphere_radii', F), ('sphere_links', U), ('skip_base', C.c_int32)]


class Config(C.Structure):
    _fields_ = [('frame_size', C.c_uint32), ('traverse_threads', C.c_uint32), ('traverse_blocks_per_sm', C.c_uint32),
                ('stream_priority', C.c_int32), ('residency_percent', C.c_uint32), ('light_steps', C.c_uint32),
                ('stage_b_form', C.c_uint32), ('stage_b_chunk', C.c_uint32), ('plain_streams', C.c_uint32),
                ('top_nodes_shared', C.c_uint32), ('sweep_unstaged', C.c_uint32),
                ('sweep_group', C.c_uint32), ('sweep_heavy_steps', C.c_uint32),
                ('sweep_descend_cap', C.c_uint32), ('sweep_heavy_wide', C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [('work_items', C.c_uint64), ('culled_items', C.c_uint64), ('fp64_retests', C.c_uint64),
                ('ms_prepare', C.c_float), ('ms_cull', C.c_float), ('ms_traverse', C.c_float),
                ('ms_total', C.c_float), ('candidates', C.c_uint64), ('exact_tests', C.c_uint64),
                ('skipped', C.c_uint64), ('node_tests', C.c_uint64), ('ms_first_pass', C.c_float),
                ('path_flags', C.c_uint32), ('first_node_tests', C.c_uint64), ('first_exact_tests', C.c_uint64),
                ('cull_sphere_tests', C.c_uint64), ('cull_sat_tests', C.c_uint64), ('deferred', C.c_uint64)]


_lib = None


def lib():
    """Load the engine.  Raises when the library has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError('librtcd_b200.so is missing: run `python -m rtcollisiondetection_b200.build` '
                               '(or __graft_entry__.build()) first')
        l = C.CDLL(LIB_PATH)
        for name in EXPORTS:
            getattr(l, name).restype = C.c_int
        _lib = l
    return _lib


def last_error():
    buf = C.create_string_buffer(1024)
    lib().rtcd_last_error(buf, C.c_size_t(1024))
    return buf.value.decode(errors='replace')


def _ok(status):
    if status != 0:
        raise RTCDError(status, last_error())


def _arr(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def _ptr(a, ct):
    if a is None:
        return None
    if hasattr(a, 'data_ptr'):            # torch tensor (device or host)
        return C.cast(C.c_void_p(a.data_ptr()), C.POINTER(ct))
    return a.ctypes.data_as(C.POINTER(ct))


def lbvh_build(ctx, lo, hi):
    """Canonical LBVH over boxes: dict(codes, perm, child[n-1, 2], node_lo, node_hi, depth)."""
    lo, hi = _arr(lo, np.float32).reshape(-1, 3), _arr(hi, np.float32).reshape(-1, 3)
    n = len(lo)
    m = max(n - 1, 1)
    out = {'codes': np.zeros(max(n, 1), np.uint32), 'perm': np.zeros(max(n, 1), np.uint32),
           'child': np.zeros((m, 2), np.uint32), 'node_lo': np.zeros((m, 3), np.float32),
           'node_hi': np.zeros((m, 3), np.float32)}
    depth = C.c_uint32()
    _ok(lib().rtcd_lbvh_build(ctx.h, _ptr(lo, C.c_float), _ptr(hi, C.c_float), C.c_uint32(n),
                              _ptr(out['codes'], C.c_uint32), _ptr(out['perm'], C.c_uint32),
                              _ptr(out['child'], C.c_uint32), _ptr(out['node_lo'], C.c_float),
                              _ptr(out['node_hi'], C.c_float), C.byref(depth)))
    for k in ('codes', 'perm'):
        out[k] = out[k][:n]
    for k in ('child', 'node_lo', 'node_hi'):
        out[k] = out[k][:max(n - 1, 0)]
    out['depth'] = depth.value
    return out


def exclusive_scan_u32(ctx, in_dev, out_dev, n, total_dev=None, stream=None):
    _ok(lib().rtcd_exclusive_scan_u32(ctx.h, _ptr(in_dev, C.c_uint32), _ptr(out_dev, C.c_uint32), C.c_uint32(n),
                                      _ptr(total_dev, C.c_uint32), C.c_void_p(stream) if stream else None))


def select_flags_u8(ctx, mask_dev, n, idx_dev, count_dev, stream=None):
    _ok(lib().rtcd_select_flags_u8(ctx.h, _ptr(mask_dev, C.c_uint8), C.c_uint32(n), _ptr(idx_dev, C.c_uint32),
                                   _ptr(count_dev, C.c_uint32), C.c_void_p(stream) if stream else None))


def loop_edges(tris):
    """Directed loop edges of a mesh as the library builds them (host only): (m, 2) uint32."""
    tris = _arr(tris, np.uint32).reshape(-1, 3)
    n = C.c_uint32()
    _ok(lib().rtcd_loop_edges(_ptr(tris, C.c_uint32), C.c_uint32(len(tris)), None, C.c_uint32(0), C.byref(n)))
    out = np.zeros((max(n.value, 1), 2), np.uint32)
    _ok(lib().rtcd_loop_edges(_ptr(tris, C.c_uint32), C.c_uint32(len(tris)), _ptr(out, C.c_uint32),
                              C.c_uint32(n.value), C.byref(n)))
    return out[:n.value]


def exact_test_probe(ctx, test, a, b):
    """The device's FP32 and FP64 results of one exact test on n pairs (numpy in, numpy out):
    test 0 segment-triangle (class, decision), 1 capsule and 2 quadratic (FP32 and FP64 distances)."""
    import torch
    a = torch.from_numpy(_arr(a, np.float32).reshape(-1, 6)).cuda()
    b = torch.from_numpy(_arr(b, np.float32).reshape(-1, 9)).cuda()
    n = a.shape[0]
    f32 = torch.zeros(max(n, 1), dtype=torch.float32, device='cuda')
    f64 = torch.zeros(max(n, 1), dtype=torch.float64, device='cuda')
    _ok(lib().rtcd_exact_test_probe(ctx.h, C.c_int(test), _ptr(a, C.c_float), _ptr(b, C.c_float), C.c_uint32(n),
                                    _ptr(f32, C.c_float), _ptr(f64, C.c_double), None))
    torch.cuda.synchronize()
    return f32.cpu().numpy()[:n], f64.cpu().numpy()[:n]


def selftest_lookback_timeout(ctx, n, spin_limit):
    """Runs the bounded-wait self-test; returns its status code (4 = RTCD_ERR_DEVICE_TIMEOUT is the
    designed outcome: every look-back wait ran out and the kernel returned)."""
    return lib().rtcd_selftest_lookback_timeout(ctx.h, C.c_uint32(n), C.c_uint32(spin_limit))


def quad_fit_weights(n_ctrl, n_wp):
    """The quadratic B-spline least-squares fit W (n_ctrl x n_wp), computed by the library (host only)."""
    out = np.zeros((n_ctrl, n_wp), np.float32)
    _ok(lib().rtcd_quad_fit_weights(C.c_uint32(n_ctrl), C.c_uint32(n_wp), _ptr(out, C.c_float)))
    return out


URDF_MAX_LINKS, URDF_NAME = 16, 128


class UrdfChain(C.Structure):
    _fields_ = [('dof', C.c_uint32), ('n_links', C.c_uint32), ('base_tf', C.c_float * 12),
                ('cos_mask', C.c_float * ((URDF_MAX_LINKS - 1) * 12)),
                ('sin_mask', C.c_float * ((URDF_MAX_LINKS - 1) * 12)),
                ('one_mask', C.c_float * ((URDF_MAX_LINKS - 1) * 12)),
                ('lower', C.c_float * (URDF_MAX_LINKS - 1)), ('upper', C.c_float * (URDF_MAX_LINKS - 1)),
                ('link_name', (C.c_char * URDF_NAME) * URDF_MAX_LINKS),
                ('link_mesh', (C.c_char * (2 * URDF_NAME)) * URDF_MAX_LINKS)]


def urdf_chain(text):
    """Parse URDF text (rtcd_urdf_chain_parse): masks, limits, link names and mesh files."""
    raw = text.encode() if isinstance(text, str) else bytes(text)
    c = UrdfChain()
    _ok(lib().rtcd_urdf_chain_parse(C.c_char_p(raw), C.c_size_t(len(raw)), C.byref(c)))
    d = c.dof
    return {'dof': d, 'base_tf': np.array(c.base_tf, np.float32),
            'cos_mask': np.array(c.cos_mask, np.float32)[:12 * d].reshape(d, 12),
            'sin_mask': np.array(c.sin_mask, np.float32)[:12 * d].reshape(d, 12),
            'one_mask': np.array(c.one_mask, np.float32)[:12 * d].reshape(d, 12),
            'lower': np.array(c.lower, np.float32)[:d], 'upper': np.array(c.upper, np.float32)[:d],
            'link_names': [c.link_name[i].value.decode() for i in range(c.n_links)],
            'link_meshes': [c.link_mesh[i].value.decode() for i in range(c.n_links)]}


def obj_load(path):
    """Load an OBJ (rtcd_obj_load): deduplicated float32 vertices [n, 3], uint32 triangles [m, 3]."""
    nv, nt = C.c_uint32(), C.c_uint32()
    p = os.fsencode(path)
    _ok(lib().rtcd_obj_load(C.c_char_p(p), None, 0, C.byref(nv), None, 0, C.byref(nt)))
    v = np.zeros((max(nv.value, 1), 3), np.float32)
    t = np.zeros((max(nt.value, 1), 3), np.uint32)
    _ok(lib().rtcd_obj_load(C.c_char_p(p), _ptr(v, C.c_float), nv, C.byref(nv), _ptr(t, C.c_uint32), nt, C.byref(nt)))
    return v[:nv.value], t[:nt.value]


def model_from_urdf(text, mesh_root):
    """A robot model dict (as Robot takes) from URDF text and the directory its
    mesh file names are relative to; links without a visual mesh get none."""
    ch = urdf_chain(text)
    V, T, voff, toff = [], [], [0], [0]
    for m in ch['link_meshes']:
        if m:
            v, t = obj_load(os.path.join(mesh_root, m))
        else:
            v, t = np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32)
        V.append(v); T.append(t)
        voff.append(voff[-1] + len(v)); toff.append(toff[-1] + len(t))
    model = {k: ch[k] for k in ('cos_mask', 'sin_mask', 'one_mask', 'base_tf', 'lower', 'upper')}
    model.update(link_verts=np.concatenate(V), link_vert_off=np.asarray(voff, np.uint32),
                 link_tris=np.concatenate(T), link_tri_off=np.asarray(toff, np.uint32), link_names=ch['link_names'])
    return model


def halton_samples(n, lower, upper, skip=0):
    """Halton roadmap samples (host): n x dim float32 in [lower, upper]."""
    lo, hi = _arr(lower, np.float32), _arr(upper, np.float32)
    out = np.zeros((max(n, 1), len(lo)), np.float32)
    _ok(lib().rtcd_halton_samples(C.c_uint32(n), C.c_uint32(len(lo)), C.c_uint32(skip), _ptr(lo, C.c_float),
                                  _ptr(hi, C.c_float), _ptr(out, C.c_float)))
    return out[:n]


def knn(ctx, points_dev, n, dim, k, idx_dev, dist_dev, weights=None, mask_dev=None, stream=None):
    """Weighted k nearest neighbours of every point (device buffers, rtcd_knn)."""
    w = _arr(weights, np.float32)
    _ok(lib().rtcd_knn(ctx.h, _ptr(points_dev, C.c_float), C.c_uint32(n), C.c_uint32(dim), _ptr(w, C.c_float),
                       C.c_uint32(k), _ptr(mask_dev, C.c_uint8), _ptr(idx_dev, C.c_uint32), _ptr(dist_dev, C.c_float),
                       C.c_void_p(stream) if stream else None))


def robot_fk(robot, q_dev, n, T_dev, stream=None):
    _ok(lib().rtcd_robot_fk(robot.h, _ptr(q_dev, C.c_float), C.c_uint32(n), _ptr(T_dev, C.c_float),
                            C.c_void_p(stream) if stream else None))


class Context:
    def __init__(self, device=0):
        self.h = VP()
        _ok(lib().rtcd_context_create(C.c_int(device), C.byref(self.h)))
        self.device = device

    def close(self):
        if self.h:
            lib().rtcd_context_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Robot:
    """Serial-chain robot: chain masks, link meshes, optional spheres."""

    def __init__(self, ctx, model, spheres=None, skip_base=True, edges=True):
        self.ctx = ctx
        m = model
        self._keep = {
            'base': _arr(m['base_tf'], np.float32), 'cos': _arr(m['cos_mask'], np.float32),
            'sin': _arr(m['sin_mask'], np.float32), 'one': _arr(m['one_mask'], np.float32),
            'lv': _arr(m['link_verts'], np.float32), 'lvo': _arr(m['link_vert_off'], np.uint32),
            'lt': _arr(m['link_tris'], np.uint32), 'lto': _arr(m['link_tri_off'], np.uint32),
            'le': _arr(m['link_edges'], np.uint32) if edges and 'link_edges' in m else None,
            'leo': _arr(m['link_edge_off'], np.uint32) if edges and 'link_edges' in m else None,
        }
        if spheres is None and 'sphere_centers' in m:
            spheres = (m['sphere_centers'], m['sphere_radii'], m['sphere_links'])
        if spheres is not None:
            self._keep['sc'] = _arr(spheres[0], np.float32)
            self._keep['sr'] = _arr(spheres[1], np.float32)
            self._keep['sl'] = _arr(spheres[2], np.uint32)
        k = self._keep
        self.dof = len(k['cos']) if k['cos'].ndim == 2 else len(k['cos']) // 12
        d = RobotDesc()
        d.dof = self.dof
        d.base_tf, d.cos_mask, d.sin_mask, d.one_mask = (_ptr(k[x], C.c_float) for x in ('base', 'cos', 'sin', 'one'))
        d.link_verts = _ptr(k['lv'], C.c_float)
        d.link_vert_offsets = _ptr(k['lvo'], C.c_uint32)
        d.link_tris = _ptr(k['lt'], C.c_uint32)
        d.link_tri_offsets = _ptr(k['lto'], C.c_uint32)
        d.link_edges = _ptr(k['le'], C.c_uint32)
        d.link_edge_offsets = _ptr(k['leo'], C.c_uint32)
        d.link_obbs = None
        if spheres is not None:
            d.n_spheres = len(k['sr'])
            d.sphere_centers = _ptr(k['sc'], C.c_float)
            d.sphere_radii = _ptr(k['sr'], C.c_float)
            d.sphere_links = _ptr(k['sl'], C.c_uint32)
        d.skip_base = 1 if skip_base else 0
        self.h = VP()
        _ok(lib().rtcd_robot_create(ctx.h, C.byref(d), C.byref(self.h)))

    def close(self):
        if self.h:
            lib().rtcd_robot_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Resident obstacle scene (triangle soup with obstacle ranges)."""

    def __init__(self, ctx, verts, tris, obstacle_tri_off=None):
        self.ctx = ctx
        v = _arr(verts, np.float32).reshape(-1, 3)
        t = _arr(tris, np.uint32).reshape(-1, 3)
        o = _arr(obstacle_tri_off, np.uint32)
        self.h = VP()
        _ok(lib().rtcd_scene_create(ctx.h, _ptr(v, C.c_float), C.c_uint32(len(v)), _ptr(t, C.c_uint32),
                                    C.c_uint32(len(t)), _ptr(o, C.c_uint32),
                                    C.c_uint32(0 if o is None else len(o) - 1), C.byref(self.h)))
        nt, ne, no = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _ok(lib().rtcd_scene_info(self.h, C.byref(nt), C.byref(ne), C.byref(no)))
        self.n_tris, self.n_edges, self.n_obstacles = nt.value, ne.value, no.value

    @classmethod
    def from_mesh(cls, ctx, mesh):
        return cls(ctx, mesh.verts, mesh.tris, mesh.obstacle_tri_off)

    def close(self):
        if self.h:
            lib().rtcd_scene_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def segment_offsets(kind, traj_off, flags=0):
    traj_off = _arr(traj_off, np.uint32)
    out = np.zeros(len(traj_off), np.uint32)
    _ok(lib().rtcd_segment_offsets(C.c_int(kind), _ptr(traj_off, C.c_uint32), C.c_uint32(len(traj_off) - 1),
                                   C.c_uint32(flags), _ptr(out, C.c_uint32)))
    return out


class Detector:
    """One detector of one kind over a robot and a scene."""

    def __init__(self, ctx, kind, robot, scene, frame_size=0, traverse_threads=0, traverse_blocks_per_sm=0,
                 stream_priority=0, residency_percent=0, light_steps=0, stage_b_form=0, stage_b_chunk=0,
                 plain_streams=0, top_nodes_shared=0, sweep_unstaged=0, sweep_group=0,
                 sweep_heavy_steps=0, sweep_descend_cap=0, sweep_heavy_wide=0):
        if isinstance(kind, str):
            kind = KIND_NAMES[kind]
        self.ctx, self.kind, self.robot, self.scene = ctx, kind, robot, scene
        cfg = Config()
        cfg.frame_size = frame_size
        cfg.traverse_threads = traverse_threads
        cfg.traverse_blocks_per_sm = traverse_blocks_per_sm
        cfg.stream_priority = stream_priority
        cfg.residency_percent = residency_percent
        cfg.light_steps = light_steps
        cfg.stage_b_form = stage_b_form
        cfg.stage_b_chunk = stage_b_chunk
        cfg.plain_streams = plain_streams
        cfg.top_nodes_shared = top_nodes_shared
        cfg.sweep_unstaged = sweep_unstaged
        cfg.sweep_group = sweep_group
        cfg.sweep_heavy_steps = sweep_heavy_steps
        cfg.sweep_descend_cap = sweep_descend_cap
        cfg.sweep_heavy_wide = sweep_heavy_wide
        self.h = VP()
        _ok(lib().rtcd_detector_create(ctx.h, C.c_int(kind), robot.h, scene.h, C.byref(cfg), C.byref(self.h)))

    @property
    def sweep(self):
        return self.kind in (LINEAR_SWEEP, QUAD_SWEEP)

    def check(self, q, traj_off=None, counts=False, segments=False, flags=0, surface=False):
        """Host-buffer call: q is a numpy array; returns dict of numpy outputs.
        surface=True: the sweeps' reference (entering-ray) semantics."""
        q = _arr(q, np.float32)
        flags |= CHECK_HOST_BUFFERS | (CHECK_COUNTS if counts else 0) | (CHECK_SURFACE if surface else 0)
        if self.sweep:
            traj_off = _arr(traj_off, np.uint32)
            n = len(traj_off) - 1
        else:
            n = len(q)
        out = {'flags': np.zeros(n, np.uint8)}
        if counts:
            out['counts'] = np.zeros(n, np.uint32)
        seg = None
        if segments:
            seg_off = segment_offsets(self.kind, traj_off, flags)
            seg = np.zeros(max(1, int(seg_off[-1])), np.uint8)
            out['seg_off'] = seg_off
        _ok(lib().rtcd_check(self.h, _ptr(q, C.c_float), _ptr(traj_off, C.c_uint32), C.c_uint32(n),
                             _ptr(out['flags'], C.c_uint8), _ptr(seg, C.c_uint8),
                             _ptr(out.get('counts'), C.c_uint32), C.c_uint32(flags), None))
        if segments:
            out['seg_flags'] = seg[:int(out['seg_off'][-1])]
        return out

    def check_device(self, q_dev, n, flags_dev, traj_off=None, counts_dev=None, seg_dev=None, flags=0, stream=None):
        """Device-buffer call (torch CUDA tensors or raw pointers); asynchronous."""
        traj_off = _arr(traj_off, np.uint32)
        if counts_dev is not None:
            flags |= CHECK_COUNTS
        _ok(lib().rtcd_check(self.h, _ptr(q_dev, C.c_float), _ptr(traj_off, C.c_uint32), C.c_uint32(n),
                             _ptr(flags_dev, C.c_uint8), _ptr(seg_dev, C.c_uint8), _ptr(counts_dev, C.c_uint32),
                             C.c_uint32(flags), C.c_void_p(stream) if stream else None))

    def sync(self, stream=None):
        _ok(lib().rtcd_sync(self.h, C.c_void_p(stream) if stream else None))

    def check_edges(self, nodes_dev, n_nodes, edges_dev, n_edges, n_wp, flags_dev, flags=0, stream=None):
        """Straight-line edges between configurations, interpolated on the device (rtcd_check_edges)."""
        _ok(lib().rtcd_check_edges(self.h, _ptr(nodes_dev, C.c_float), C.c_uint32(n_nodes), _ptr(edges_dev, C.c_uint32),
                                   C.c_uint32(n_edges), C.c_uint32(n_wp), _ptr(flags_dev, C.c_uint8), C.c_uint32(flags),
                                   C.c_void_p(stream) if stream else None))

    def autotune(self, q_dev, n, traj_off=None, stream=None):
        """Pick the fastest traversal launch shape on this device-resident batch."""
        traj_off = _arr(traj_off, np.uint32)
        best = Config()
        ms = C.c_float()
        _ok(lib().rtcd_detector_autotune(self.h, _ptr(q_dev, C.c_float), _ptr(traj_off, C.c_uint32), C.c_uint32(n),
                                         C.c_void_p(stream) if stream else None, C.byref(best), C.byref(ms)))
        return {'traverse_threads': best.traverse_threads, 'traverse_blocks_per_sm': best.traverse_blocks_per_sm,
                'light_steps': best.light_steps, 'stage_b_form': best.stage_b_form,
                'stage_b_chunk': best.stage_b_chunk, 'top_nodes_shared': best.top_nodes_shared,
                'sweep_unstaged': best.sweep_unstaged, 'sweep_group': best.sweep_group,
                'sweep_descend_cap': best.sweep_descend_cap, 'sweep_heavy_wide': best.sweep_heavy_wide,
                'traverse_ms': ms.value}

    def stats(self):
        s = Stats()
        _ok(lib().rtcd_last_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_ if not k.startswith('reserved')}

    def close(self):
        if self.h:
            lib().rtcd_detector_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CollisionDetector:
    """Mirror of the upstream ``RTCD::CollisionDetector`` call sequence.

    ``setupScene(scene)``, ``setupRobot(robot)``, ``setupOptix()`` and
    ``buildSBT()`` are accepted for drop-in call order (the last two have
    nothing to do here); ``prepareUpdateData(poses, n)`` stages host poses
    (``CCRobotWrapper.h:39-46``), ``setNCheck(n)`` sets the query size
    (``CollisionDetector.h:354``), ``check()`` runs it and ``downloadResult``
    returns the per-pose (per-trajectory) upstream hit counts, nonzero = hit
    (``CollisionDetector.h:62``).  The curve detectors follow the reference's
    semantics (loop edges entering a swept piece, RTCD_CHECK_SURFACE) unless
    ``solid_sweeps`` is set.
    """

    def __init__(self, ctx, kind, robot=None, scene=None, solid_sweeps=False):
        self.ctx, self.kind = ctx, KIND_NAMES.get(kind, kind)
        self.robot, self.scene, self.det = robot, scene, None
        self.poses, self.traj_off, self.n = None, None, 0
        self.result = None
        self.solid_sweeps = solid_sweeps

    def setupScene(self, scene):
        self.scene = scene
        self.det = None

    def setupRobot(self, robot):
        self.robot = robot
        self.det = None

    def setupOptix(self):
        pass

    def buildSBT(self):
        if self.det is None:
            self.det = Detector(self.ctx, self.kind, self.robot, self.scene)

    def prepareUpdateData(self, poses, n, traj_off=None):
        self.poses, self.traj_off = np.ascontiguousarray(poses, np.float32), traj_off
        self.n = n

    def setNCheck(self, n):
        self.n = n

    def check(self):
        self.buildSBT()
        if self.det.sweep:
            traj = np.asarray(self.traj_off[:self.n + 1], np.uint32)
            self.result = self.det.check(self.poses, traj, counts=True, surface=not self.solid_sweeps)
        else:
            self.result = self.det.check(self.poses[:self.n], counts=True)

    def downloadResult(self):
        return self.result['counts'].copy()

    def flags(self):
        return self.result['flags'].copy()

    def clearResult(self):
        self.result = None


class ServerConfig(C.Structure):
    _fields_ = [('slots', C.c_uint32), ('max_batch_units', C.c_uint32), ('memory_budget', C.c_uint64),
                ('fast_slots', C.c_uint32), ('fast_max_units', C.c_uint32), ('bulk_share', C.c_uint32),
                ('reserved', C.c_uint32 * 1)]


class ServerStats(C.Structure):
    _fields_ = [('submitted', C.c_uint64), ('completed', C.c_uint64), ('failed', C.c_uint64),
                ('units_completed', C.c_uint64), ('batches', C.c_uint64), ('inflight_bytes_peak', C.c_uint64),
                ('queue_depth', C.c_uint32), ('reserved0', C.c_uint32), ('p50_ms', C.c_double),
                ('p99_ms', C.c_double), ('mean_ms', C.c_double), ('max_ms', C.c_double),
                ('queue_p50_ms', C.c_double), ('queue_p99_ms', C.c_double), ('run_p99_ms', C.c_double),
                ('workspace_grows', C.c_uint64), ('grow_ms', C.c_double), ('run_max_ms', C.c_double),
                ('run_max_kind', C.c_uint32), ('run_max_units', C.c_uint32), ('run_max_grows', C.c_uint32),
                ('run_max_slot', C.c_uint32), ('run_max_at_s', C.c_double)]


class Server:
    """Continuous-batching request server (rtcd_server_*): submit from any
    thread, wait for tickets; requests for the same detector are merged into
    shared launches across ``slots`` concurrent streams."""

    def __init__(self, ctx, slots=4, max_batch_units=65536, memory_budget=0, fast_slots=0, fast_max_units=0,
                 bulk_share=0):
        cfg = ServerConfig()
        cfg.slots, cfg.max_batch_units, cfg.memory_budget = slots, max_batch_units, memory_budget
        cfg.fast_slots, cfg.fast_max_units, cfg.bulk_share = fast_slots, fast_max_units, bulk_share
        self.ctx = ctx
        self.h = VP()
        _ok(lib().rtcd_server_create(ctx.h, C.byref(cfg), C.byref(self.h)))
        self._meta = {}

    def prepare(self, det, max_units=0):
        """Size every slot's workspace for `det` up front (serving then never allocates)."""
        _ok(lib().rtcd_server_prepare(self.h, det.h, C.c_uint32(max_units)))

    def submit(self, det, q, traj_off=None, counts=False, endpoints=True, surface=False):
        q = _arr(q, np.float32)
        flags = (CHECK_COUNTS if counts else 0) | (0 if endpoints else CHECK_NO_ENDPOINTS) | \
            (CHECK_SURFACE if surface else 0)
        if det.sweep:
            traj_off = _arr(traj_off, np.uint32)
            n = len(traj_off) - 1
            segs = int(segment_offsets(det.kind, traj_off, flags)[-1])
        else:
            n, segs = len(q), 0
        t = C.c_uint64()
        _ok(lib().rtcd_server_submit(self.h, det.h, _ptr(q, C.c_float), _ptr(traj_off, C.c_uint32), C.c_uint32(n),
                                     C.c_uint32(flags), C.byref(t)))
        self._meta[t.value] = (n, segs, counts)
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        n, segs, counts = self._meta[ticket]
        out = {'flags': np.zeros(max(n, 1), np.uint8)}
        seg = np.zeros(max(segs, 1), np.uint8) if segs else None
        cnt = np.zeros(max(n, 1), np.uint32) if counts else None
        lat = C.c_double()
        _ok(lib().rtcd_server_wait(self.h, C.c_uint64(ticket), C.c_int32(timeout_ms), _ptr(out['flags'], C.c_uint8),
                                   _ptr(seg, C.c_uint8), _ptr(cnt, C.c_uint32), C.byref(lat)))
        del self._meta[ticket]
        out['flags'] = out['flags'][:n]
        if seg is not None:
            out['seg_flags'] = seg[:segs]
        if cnt is not None:
            out['counts'] = cnt[:n]
        out['latency_ms'] = lat.value
        return out

    def stats(self):
        s = ServerStats()
        _ok(lib().rtcd_server_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_ if not k.startswith('reserved')}

    def reset_stats(self):
        _ok(lib().rtcd_server_reset_stats(self.h))

    def close(self):
        if self.h:
            lib().rtcd_server_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
