"""Benchmark of the batched collision-query path on B200.

Workload (one step): the RobotToObs detector over 65,536 uniform random
Panda poses against the dense synthetic scene (64 boxes, 256 level-3
icospheres, one 100k-triangle noisy sphere: 428,448 triangles), flags out.
``--config`` selects the other workloads (ObsToRobot small/dense, linear and
quadratic sweeps) for the same measurement.

Timing: W untimed warm-up steps, then K steps; a 256 MiB buffer is written
before every step to flush the 126 MB L2 and each step is timed with CUDA
events on the launching stream (max over ranks for N > 1, weak scaling:
every rank checks its own batch).  ``e2e`` repeats the step through the
public C ABI with host buffers (pose upload and flag download inside the
timed call; the step replayed as one CUDA graph that holds the copies
between the pinned staging and the device, unless ``--no-graph``).
``plain`` is the same engine driven the upstream way: frames of 1,024 poses
round-robin over 4 streams, one host thread per stream, the culled item count
read back per frame (``plain_frame64``: 64-pose frames on one stream).
``cpu_baseline`` times the FP64 oracle (flags only, every host thread) on a
bounded sample.

``--impl reference`` times the CPU restatement of the reference path (the
oracle port; the upstream OptiX path needs RT cores and the OptiX SDK) on the
same workload and prints the same JSON line with ``"impl": "reference"``.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'poses/s and p50/p99 latency: batched-served vs plain, same B200, 0 flag errors'
PEAK_FALLBACK = {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}


def load_peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        d = json.load(open(p))
        return d, 'measured'
    return dict(PEAK_FALLBACK), 'fallback'


CONFIGS = {
    'c2': dict(kind='RobotToObs', n=65536, scene='dense',
               workload='RobotToObs, 65,536 uniform Panda poses, dense scene 64 boxes + 256 level-3 icospheres + '
                        '100k-tri noisy sphere (428,448 tris) over x,y in [-1.5,1.5] m, z in [0,1.5] m'),
    'c2o': dict(kind='ObsToRobot', n=65536, scene='dense',
                workload='ObsToRobot, 65,536 uniform Panda poses, dense 428,448-tri scene'),
    'c1': dict(kind='ObsToRobot', n=1024, scene='small',
               workload='ObsToRobot, 1,024 uniform Panda poses, 12 boxes + 16 level-2 icospheres (5,264 tris)'),
    'c3': dict(kind='Linear', n=4096, scene='sweep', wp=32,
               workload='Linear sweep, 4,096 random-walk trajectories x 32 waypoints, 64 spheres, 49,744-tri scene'),
    'c4': dict(kind='Quadratic', n=4096, scene='sweep', wp=(8, 64),
               workload='Quadratic sweep, 4,096 trajectories of 8-64 waypoints (log-uniform), 64 spheres, '
                        '49,744-tri scene'),
    'c2_200k': dict(kind='RobotToObs', n=65536, scene='dense200k',
                    workload='RobotToObs, 65,536 uniform Panda poses, dense scene with level-2 icospheres '
                             '(64 boxes + 256 level-2 icospheres + 100k-tri noisy sphere, 182,688 tris)'),
    'c2_cube': dict(kind='RobotToObs', n=65536, scene='dense_cube',
                    workload='RobotToObs, 65,536 uniform Panda poses, the dense composition (428,448 tris) packed '
                             'into the 1 m workspace cube in front of the robot (box extents U(0.02, 0.6) m)'),
    'c3s': dict(kind='Linear', n=4096, scene='sweep_sparse', wp=32,
                workload='Linear sweep, 4,096 random-walk trajectories x 32 waypoints, 64 spheres, sparse '
                         '48,784-tri scene (12 boxes + 38 level-3 icospheres; ~40 % of trajectories collide)'),
    'c4s': dict(kind='Quadratic', n=4096, scene='sweep_sparse', wp=(8, 64),
                workload='Quadratic sweep, 4,096 trajectories of 8-64 waypoints (log-uniform), 64 spheres, '
                         'sparse 48,784-tri scene'),
    # the reference's own benchmark shelves (models/curobo, placements of its scene headers), batch 4096
    'ref_simple_r2o': dict(kind='RobotToObs', n=4096, scene='ref_simple',
                           workload='RobotToObs, 4,096 uniform poses, reference simple shelf (15,008 tris)'),
    'ref_simple_o2r': dict(kind='ObsToRobot', n=4096, scene='ref_simple',
                           workload='ObsToRobot, 4,096 uniform poses, reference simple shelf (15,008 tris)'),
    'ref_medium_r2o': dict(kind='RobotToObs', n=4096, scene='ref_medium',
                           workload='RobotToObs, 4,096 uniform poses, reference medium shelf (71,746 tris)'),
    'ref_medium_o2r': dict(kind='ObsToRobot', n=4096, scene='ref_medium',
                           workload='ObsToRobot, 4,096 uniform poses, reference medium shelf (71,746 tris)'),
    'ref_dense_r2o': dict(kind='RobotToObs', n=4096, scene='ref_dense',
                          workload='RobotToObs, 4,096 uniform poses, reference dense shelf (202,330 tris)'),
    'ref_dense_o2r': dict(kind='ObsToRobot', n=4096, scene='ref_dense',
                          workload='ObsToRobot, 4,096 uniform poses, reference dense shelf (202,330 tris)'),
    'ref_dense_linear': dict(kind='Linear', n=4096, scene='ref_dense', wp=16,
                             workload='Linear sweep, 4,096 trajectories x 16 waypoints, reference dense shelf'),
    'ref_dense_quad': dict(kind='Quadratic', n=4096, scene='ref_dense', wp=(8, 16),
                           workload='Quadratic sweep, 4,096 trajectories of 8-16 waypoints (4-8 control points), '
                                    'reference dense shelf'),
}


def make_inputs(cfg, rank, scenes):
    model = scenes.load_panda()
    if cfg['scene'].startswith('ref_'):
        mesh = scenes.reference_scene(cfg['scene'][4:])
    else:
        mesh = {'dense': scenes.discrete_dense, 'small': scenes.discrete_small,
                'dense200k': lambda: scenes.discrete_dense(ico_level=2), 'dense_cube': scenes.discrete_dense_cube,
                'sweep': scenes.sweep_scene, 'sweep_sparse': scenes.sweep_scene_sparse}[cfg['scene']]()
    spheres = scenes.synth_spheres(model) if cfg['kind'] in ('Linear', 'Quadratic') else None
    if cfg['kind'] in ('Linear', 'Quadratic'):
        wp = cfg['wp']
        counts = wp if np.isscalar(wp) else scenes.log_uniform_counts(cfg['n'], wp[0], wp[1], seed=rank)
        q, off = scenes.random_walk_trajectories(model, cfg['n'], counts, seed=rank)
    else:
        q, off = scenes.uniform_poses(model, cfg['n'], seed=rank), None
    return model, mesh, spheres, q, off


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 20 ms."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc, self.pre = gpu, [], None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '20'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 3.0:   # sampling is running before the timed region
                time.sleep(0.01)
            self.pre = self.rows[-1:]
            self.rows.clear()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def stop(self):
        bracketed = False
        if self.proc and not self.rows:
            # a timed region shorter than the sampling interval: bracket it with the sample just
            # before it and the first one after it
            t0 = time.time()
            while not self.rows and time.time() - t0 < 1.0:
                time.sleep(0.002)
            self.rows[:0] = self.pre
            bracketed = True
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if not self.rows:
            return None
        sm = [float(r[1]) for r in self.rows if r[1].replace('.', '', 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace('.', '', 1).isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and 'Active' in r[5 + k]
                          and 'Not' not in r[5 + k]})
        out = {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
               'reasons': reasons, 'samples': len(self.rows)}
        if bracketed:
            out['note'] = 'timed region shorter than the 20 ms sampling interval: samples just before and after it'
        return out


def cpu_baseline(cfg, model, mesh, spheres, q, off, seconds=10.0):
    """The oracle (FP64, flags only for the discrete kinds) on a bounded sample."""
    from oracle import oracle as O
    robot = O.Robot(model, spheres=spheres)
    scene = O.Scene(mesh)
    threads = os.cpu_count() or 1
    if cfg['kind'] in ('RobotToObs', 'ObsToRobot'):
        prep = O.PreparedDiscrete(O.ROBOT_TO_OBS if cfg['kind'] == 'RobotToObs' else O.OBS_TO_ROBOT, robot, scene)
        n = 256
        while True:
            t0 = time.perf_counter()
            prep.flags(q[:n], threads)
            dt = time.perf_counter() - t0
            if dt * 4 > seconds or n >= len(q):
                break
            n = min(len(q), n * 4)
        unit, value = 'poses/s', n / dt
        sample = '%d of the %d poses, flags only with per-pose early exit' % (n, len(q))
    else:
        quad = cfg['kind'] == 'Quadratic'
        n = 16
        while True:
            t0 = time.perf_counter()
            O.sweep(quad, robot, scene, q[:off[n]], off[:n + 1], threads=threads)
            dt = time.perf_counter() - t0
            if dt * 4 > seconds or n >= len(off) - 1:
                break
            n = min(len(off) - 1, n * 4)
        unit, value = 'trajectories/s', n / dt
        sample = '%d of the %d trajectories, full segment flags' % (n, len(off) - 1)
    return {'value': value, 'unit': unit, 'cores': threads, 'kind': 'port', 'sample': sample,
            'seconds': round(dt, 3)}


def oracle_errors(cfg, model, mesh, spheres, q, off, flags, n_sample=512, two_way=False, containment=False):
    """Flag mismatches outside the 1e-5 m band on a sample of the batch."""
    from oracle import oracle as O
    robot = O.Robot(model, spheres=spheres)
    scene = O.Scene(mesh)
    if cfg['kind'] in ('RobotToObs', 'ObsToRobot'):
        k = O.ROBOT_TO_OBS if cfg['kind'] == 'RobotToObs' else O.OBS_TO_ROBOT
        idx = np.linspace(0, len(q) - 1, min(n_sample, len(q))).astype(int)
        ref = O.discrete(k, robot, scene, q[idx])
        hit, band = ref['hit'].copy(), ref['band'].copy()
        if two_way:
            other = O.discrete(1 - k, robot, scene, q[idx])
            hit |= other['hit']
            band |= other['band']
        want = hit.astype(np.uint8)
        if containment:
            cont = O.containment(robot, scene, q[idx], skip=hit)
            want |= 2 * cont['contain']
            band |= cont['band']
        err = int(((flags[idx] != want) & (band == 0)).sum())
        return {'flag_errors': err, 'checked': len(idx), 'in_band': int(band.sum()),
                'collision_rate': float((want != 0).mean())}
    m = min(len(off) - 1, n_sample // 4)
    ref = O.sweep(cfg['kind'] == 'Quadratic', robot, scene, q[:off[m]], off[:m + 1])
    err = int(((flags[:m] != ref['traj_hit']) & (ref['traj_band'] == 0)).sum())
    return {'flag_errors': err, 'checked': m, 'in_band': int(ref['traj_band'].sum()),
            'collision_rate': float(ref['traj_hit'].mean())}


def served_stream(ctx, seconds, rate=2000.0, seed=0, slots=4, plain_seconds=1.0, server_kw=None, details=False,
                  saturate_requests=0):
    """Mixed request stream against three resident scenes (5k, 50k, ~500k
    triangles): Poisson arrivals at `rate` req/s for `seconds`; half discrete
    RobotToObs batches of log-uniform[1, 4096] poses, half continuous batches
    (linear / quadratic alternately) of log-uniform[1, 1024] trajectories with
    log-uniform[8, 128] waypoints.  Requests go to the continuous-batching
    server from a submitter thread at their arrival times; latency is submit
    to result.  The same arrivals (first `plain_seconds`) are then replayed on
    the plain form - one request at a time, each a frame-by-frame check with a
    host round trip per frame - for comparison.  With saturate_requests, the
    first that many requests of the mix are also submitted all at once (no
    arrival gaps), and the units the server completes per second are set
    beside the plain form's on the same requests (saturated throughput, not
    the offered load)."""
    import threading
    from rtcollisiondetection_b200 import rtcd, scenes
    model = scenes.load_panda()
    sph = scenes.synth_spheres(model)
    robot = rtcd.Robot(ctx, model, spheres=sph)
    meshes = [scenes.discrete_small(), scenes.sweep_scene(), scenes.served_large_scene()]
    scn = [rtcd.Scene.from_mesh(ctx, m) for m in meshes]
    dets = [{k: rtcd.Detector(ctx, k, robot, s) for k in ('RobotToObs', 'Linear', 'Quadratic')} for s in scn]
    rng = np.random.default_rng(seed)
    n_req = int(rate * seconds)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    pose_pool = scenes.uniform_poses(model, 1 << 17, seed=seed + 1)
    traj_q, traj_off = scenes.random_walk_trajectories(model, 2048, scenes.log_uniform_counts(2048, 8, 128, seed=seed + 2),
                                                       seed=seed + 3)
    reqs = []
    for i in range(n_req):
        s = int(rng.integers(0, 3))
        if rng.random() < 0.5:
            n = int(np.rint(np.exp(rng.uniform(0, np.log(4096)))))
            a = int(rng.integers(0, len(pose_pool) - n))
            reqs.append((dets[s]['RobotToObs'], pose_pool[a:a + n], None, n))
        else:
            k = 'Linear' if rng.random() < 0.5 else 'Quadratic'
            nt = int(np.rint(np.exp(rng.uniform(0, np.log(1024)))))
            t0 = int(rng.integers(0, 2048 - nt + 1))
            off = traj_off[t0:t0 + nt + 1] - traj_off[t0]
            reqs.append((dets[s][k], traj_q[traj_off[t0]:traj_off[t0 + nt]], off, nt))

    def run_server():
        server = rtcd.Server(ctx, slots=slots, **(server_kw or {}))
        for d in dets:              # every slot's workspace sized outside the measured window
            for det in d.values():
                server.prepare(det, 1 << 17 if det.sweep else 0)
        server.reset_stats()
        tickets = [None] * n_req
        lat = np.zeros(n_req)
        start = time.perf_counter()

        def submitter():
            for i, (det, q, off, n) in enumerate(reqs):
                delay = arrivals[i] - (time.perf_counter() - start)
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = server.submit(det, q, off)

        th = threading.Thread(target=submitter)
        th.start()
        for i in range(n_req):
            while tickets[i] is None:
                time.sleep(0.0002)
            lat[i] = server.wait(tickets[i])['latency_ms']
        th.join()
        wall = time.perf_counter() - start
        st = server.stats()
        server.close()
        return lat, wall, st

    lat, wall, st = run_server()

    def saturated(m):
        """Units per second (poses + trajectories) of the first m requests, all submitted at once to
        the server, and the same requests checked one at a time on the plain form."""
        server = rtcd.Server(ctx, slots=slots, **(server_kw or {}))
        for d in dets:
            for det in d.values():
                server.prepare(det, 1 << 17 if det.sweep else 0)
        units = float(sum(r[3] for r in reqs[:m]))
        t0 = time.perf_counter()
        tickets = [server.submit(det, q, off) for det, q, off, _ in reqs[:m]]
        for t in tickets:
            server.wait(t)
        sw = time.perf_counter() - t0
        server.close()
        t0 = time.perf_counter()
        for det, q, off, _ in reqs[:m]:
            det.check(q, off, flags=0 if det.sweep else rtcd.CHECK_PLAIN)
        pw = time.perf_counter() - t0
        return {'requests': m, 'units': units, 'served_units_per_s': units / sw, 'served_wall_s': sw,
                'plain_units_per_s': units / pw, 'plain_wall_s': pw, 'served_over_plain': pw / sw,
                'note': 'units = poses + trajectories of the mixed requests; served = all submitted at once, '
                        'continuous batching over 4 slots; plain = one request at a time (discrete requests on '
                        'the upstream-shaped frame path, sweep requests as one call each)'}

    sat = saturated(min(saturate_requests, n_req)) if saturate_requests > 0 else None
    disc = np.array([r[2] is None for r in reqs])
    sizes = np.array([r[3] for r in reqs])
    poses = int(sizes[disc].sum())
    trajs = int(sizes[~disc].sum())
    out = {'seconds': seconds, 'rate_req_s': rate, 'requests': n_req, 'slots': slots, 'wall_s': wall,
           'p50_ms_discrete_le4096': float(np.percentile(lat[disc], 50)),
           'p99_ms_discrete_le4096': float(np.percentile(lat[disc], 99)),
           'p50_ms_all': float(np.percentile(lat, 50)), 'p99_ms_all': float(np.percentile(lat, 99)),
           'poses_per_s': poses / wall, 'trajectories_per_s': trajs / wall, 'batches': st['batches'],
           'queue_p50_ms': st['queue_p50_ms'], 'queue_p99_ms': st['queue_p99_ms'], 'run_p99_ms': st['run_p99_ms'],
           'workspace_grows': st['workspace_grows'], 'grow_ms': st['grow_ms'],
           'longest_launch': {'ms': st['run_max_ms'], 'at_s': st['run_max_at_s'], 'slot': st['run_max_slot'],
                              'kind': ['ObsToRobot', 'RobotToObs', 'Linear', 'Quadratic'][st['run_max_kind']],
                              'units': st['run_max_units'], 'grows': st['run_max_grows']},
           'scenes_tris': [m.n_tris for m in meshes],
           'p99_margin_ms_discrete_le4096': 2.0 - float(np.percentile(lat[disc], 99)),
           'p99_margin_ms_all': 2.0 - float(np.percentile(lat, 99))}
    if sat:
        out['saturated'] = sat
    # the slowest requests: what they were and when they arrived (tail diagnosis)
    scene_of = {id(det): i for i, d in enumerate(dets) for det in d.values()}
    worst = np.argsort(-lat)[:8]
    out['slowest'] = [{'ms': round(float(lat[i]), 3), 'arrival_s': round(float(arrivals[i]), 3),
                       'kind': ['ObsToRobot', 'RobotToObs', 'Linear', 'Quadratic'][reqs[i][0].kind],
                       'units': int(reqs[i][3]), 'scene': scene_of[id(reqs[i][0])]} for i in worst]
    if details:
        out['details'] = {'latency_ms': lat, 'discrete': disc, 'size': sizes,
                          'scene': np.array([scene_of[id(r[0])] for r in reqs]),
                          'kind': [r[0].kind for r in reqs]}
    if plain_seconds <= 0:
        return out
    # plain: the same arrivals, one request at a time through the frame-by-frame path
    m = int(rate * plain_seconds)
    plat = np.zeros(m)
    start = time.perf_counter()
    for i in range(m):
        det, q, off, n = reqs[i]
        delay = arrivals[i] - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        det.check(q, off, flags=0 if det.sweep else rtcd.CHECK_PLAIN)
        plat[i] = (time.perf_counter() - start - arrivals[i]) * 1e3
    pwall = time.perf_counter() - start
    pd = disc[:m]
    out['plain'] = {'requests': m, 'wall_s': pwall, 'p50_ms_discrete_le4096': float(np.percentile(plat[pd], 50)),
                    'p99_ms_discrete_le4096': float(np.percentile(plat[pd], 99)),
                    'poses_per_s': float(sizes[:m][pd].sum() / pwall)}
    return out


def fp64_statement(cfg, ctx, model, mesh, spheres, q, off, n_pairs=4096, seed=0):
    """The error of the FP32 exact tests against FP64, on near-degenerate pairs
    drawn from this workload's own geometry, run through the device's own
    arithmetic (rtcd_exact_test_probe) and checked against the oracle on the
    same float inputs.

    Discrete: segments crossing scene triangles within 1e-7..1e-5 m of an
    edge, a vertex or the plane: how many the FP32 filter hands to FP64, and
    how many of its certain decisions (or the FP64 re-test's) disagree with
    the oracle where the oracle's margin exceeds 1e-12 m (both must be 0).
    Sweeps: segments passing within +-20 um of the radius of the workload's
    own pieces (capsules or quadratic Bezier pieces): the largest FP32 and FP64
    distance errors against the oracle's FP64 branch and bound, and the count
    of FP32 sides wrong outside the FP64 re-test band (must be 0)."""
    from oracle import oracle as O
    from rtcollisiondetection_b200 import rtcd
    rng = np.random.default_rng(seed)
    if cfg['kind'] in ('RobotToObs', 'ObsToRobot'):
        tri = mesh.verts[mesh.tris[rng.integers(0, len(mesh.tris), n_pairs)]].astype(np.float64)  # n x 3 x 3
        nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        mode = rng.integers(0, 3, n_pairs)        # 0 near an edge, 1 near a vertex, 2 endpoint near the plane
        delta = rng.choice([-1e-5, -1e-6, -1e-7, 1e-7, 1e-6, 1e-5], n_pairs)
        k = rng.integers(0, 3, n_pairs)
        a, b = tri[np.arange(n_pairs), k], tri[np.arange(n_pairs), (k + 1) % 3]
        c = tri[np.arange(n_pairs), (k + 2) % 3]
        t = rng.uniform(0.1, 0.9, n_pairs)[:, None]
        on_edge = a + t * (b - a)
        inward = c - on_edge - ((c - on_edge) * (b - a)).sum(1, keepdims=True) / ((b - a) ** 2).sum(1, keepdims=True) * (b - a)
        inward /= np.linalg.norm(inward, axis=1, keepdims=True)
        x = np.where((mode == 0)[:, None], on_edge + delta[:, None] * inward,
                     np.where((mode == 1)[:, None], a + delta[:, None] * inward, tri.mean(1)))
        L = 0.01
        p = x - L * nrm
        qq = x + np.where((mode == 2)[:, None], delta[:, None], L) * nrm
        seg = np.concatenate([p, qq], 1).astype(np.float32)
        trif = tri.reshape(n_pairs, 9).astype(np.float32)
        cls, dec = rtcd.exact_test_probe(ctx, 0, seg, trif)
        wrong32 = wrong64 = margin_ok = 0
        for i in range(n_pairs):
            s64 = seg[i].astype(np.float64)
            t64 = trif[i].astype(np.float64)
            hit, m = O.seg_tri(s64[:3], s64[3:], t64[:3], t64[3:6], t64[6:])
            if m <= 1e-12:
                continue
            margin_ok += 1
            if cls[i] != 2 and bool(cls[i]) != hit:
                wrong32 += 1
            if bool(dec[i]) != hit:
                wrong64 += 1
        return {'test': 'segment-triangle', 'pairs': n_pairs, 'decided_by_oracle': margin_ok,
                'fp32_undecided': int((cls == 2).sum()), 'fp32_certain_wrong': wrong32, 'fp64_wrong': wrong64,
                'sample': 'segments crossing the scene\'s own triangles within 1e-7..1e-5 m of an edge, a vertex '
                          'or the plane'}
    # sweeps: pieces of the first trajectories of this batch
    quad = cfg['kind'] == 'Quadratic'
    nt = min(64, len(off) - 1)
    T = O.fk(model, q[:off[nt]])                            # FP64 link transforms per waypoint
    cen, rad, lnk = spheres[0].astype(np.float64), spheres[1].astype(np.float64), spheres[2]
    segs, pieces, rs = [], [], []
    for i in range(n_pairs):
        tr = int(rng.integers(0, nt))
        w0, nw = int(off[tr]), int(off[tr + 1] - off[tr])
        sph = int(rng.integers(0, len(rad)))
        P = np.stack([T[w0 + w, lnk[sph]].reshape(3, 4) @ np.append(cen[sph], 1.0) for w in range(nw)])
        if quad:
            nc = O.quad_ctrl_count(nw)
            C = O.fit_weights(nc, nw) @ P
            g = int(rng.integers(0, nc - 2))
            B = np.stack([(C[g] + C[g + 1]) / 2, C[g + 1], (C[g + 1] + C[g + 2]) / 2])
        else:
            g = int(rng.integers(0, nw - 1))
            B = np.stack([P[g], P[g + 1], P[g + 1]])
        B = B.astype(np.float32).astype(np.float64)
        u = rng.uniform(0, 1)
        pt = (1 - u) ** 2 * B[0] + 2 * u * (1 - u) * B[1] + u ** 2 * B[2]
        tg = 2 * (1 - u) * (B[1] - B[0]) + 2 * u * (B[2] - B[1])
        if np.linalg.norm(tg) < 1e-9:   # a sphere that does not move (base link): any direction
            tg = rng.normal(size=3)
        tg = tg / np.linalg.norm(tg)
        nv = np.cross(tg, rng.normal(size=3))
        nv /= np.linalg.norm(nv)
        ev = np.cross(nv, tg) if rng.random() < 0.5 else tg
        r = float(rad[sph])
        x = pt + (r + rng.uniform(-2e-5, 2e-5)) * nv
        segs.append(np.concatenate([x - 0.02 * ev, x + 0.02 * ev]))
        pieces.append(B.reshape(9))
        rs.append(r)
    seg = np.array(segs, np.float32)
    pc = np.array(pieces, np.float32)
    d32, d64 = rtcd.exact_test_probe(ctx, 2 if quad else 1, seg, pc)
    ref = np.array([O.seg_quad(seg[i, :3], seg[i, 3:], pc[i, :3], pc[i, 3:6], pc[i, 6:]) if quad else
                    O.seg_seg(seg[i, :3], seg[i, 3:], pc[i, :3], pc[i, 3:6]) for i in range(n_pairs)])
    rs = np.array(rs)
    band = 2e-6 + 1e-6 * rs
    outside = np.abs(ref - rs) > band
    wrong = int((((d32 <= rs) != (ref <= rs)) & outside).sum())
    return {'test': 'segment-quadratic piece' if quad else 'segment-capsule', 'pairs': n_pairs,
            'max_abs_err_fp32_m': float(np.abs(d32 - ref).max()), 'max_abs_err_fp64_m': float(np.abs(d64 - ref).max()),
            'in_fp64_band': int((~outside).sum()), 'fp32_side_wrong_outside_band': wrong,
            'sample': 'segments within +-20 um of the radius of this batch\'s own %s' % (
                'quadratic pieces (fitted control points)' if quad else 'capsules')}


FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # nominal: SMs x FP32 lanes x FMA x max SM clock


def fp32_work(cfg, model, mesh, spheres, q, off, scene, t_trav_ms, sample=256):
    """FP32 work of the reference algorithm for this batch, from the FP64 oracle's
    canonical-LBVH counters on a sample (full traversal, no early exit, no OBB
    cull - an upper bound), weighted 18 flops per node slab test, 40 per
    segment-triangle, 45 per segment-capsule, 200 per segment-quadratic test,
    72 per link of FK and 36 per moved edge; scaled to the batch and divided
    by the traversal span."""
    from oracle import oracle as O
    robot = O.Robot(model, spheres=spheres)
    oscene = O.Scene(mesh)
    links = model['cos_mask'].shape[0] + 1
    if cfg['kind'] in ('RobotToObs', 'ObsToRobot'):
        k = O.ROBOT_TO_OBS if cfg['kind'] == 'RobotToObs' else O.OBS_TO_ROBOT
        idx = np.linspace(0, len(q) - 1, min(sample, len(q))).astype(int)
        w = O.discrete(k, robot, oscene, q[idx], work=True)
        edges = int(model['link_edge_off'][-1] - model['link_edge_off'][1]) if k == O.ROBOT_TO_OBS else 0
        per_unit = (18.0 * w['node_tests'].mean() + 40.0 * w['prim_tests'].mean() + 72.0 * links + 36.0 * edges)
        units = len(q)
    else:
        m = min(len(off) - 1, sample // 4)
        w = O.sweep(cfg['kind'] == 'Quadratic', robot, oscene, q[:off[m]], off[:m + 1], work=True)
        wpt = float(off[m]) / m
        per_unit = (18.0 * w['node_tests'].mean() + (200.0 if cfg['kind'] == 'Quadratic' else 45.0)
                    * w['prim_tests'].mean() + 72.0 * links * wpt)
        units = len(off) - 1
    tflops = per_unit * units / (t_trav_ms / 1e3) / 1e12
    return {'rate': tflops, 'unit': 'TFLOP/s', 'flops_per_unit': per_unit,
            'note': 'the reference algorithm (every edge ray traversed to the end) would need this many flops at '
                    'this speed; early exit and the OBB cull skip most of it, so it can exceed the peak',
            'sample': 'oracle counters over %d of %d units' % (len(idx) if cfg['kind'] in ('RobotToObs', 'ObsToRobot')
                                                              else m, units)}


def run_reference(args, cfg, rank, world):
    from rtcollisiondetection_b200 import scenes
    if rank != 0:
        return
    model, mesh, spheres, q, off = make_inputs(cfg, 0, scenes)
    from oracle import oracle as O
    robot = O.Robot(model, spheres=spheres)
    scene = O.Scene(mesh)
    threads = os.cpu_count() or 1
    discrete = cfg['kind'] in ('RobotToObs', 'ObsToRobot')
    if discrete:
        prep = O.PreparedDiscrete(O.ROBOT_TO_OBS if cfg['kind'] == 'RobotToObs' else O.OBS_TO_ROBOT, robot, scene)
        sample = max(256, min(len(q), args.ref_sample))

        def step():
            prep.flags(q[:sample], threads)
        units = sample
    else:
        quad = cfg['kind'] == 'Quadratic'
        sample = max(4, min(len(off) - 1, args.ref_sample // 64))

        def step():
            O.sweep(quad, robot, scene, q[:off[sample]], off[:sample + 1], threads=threads)
        units = sample
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    unit = 'poses/s' if discrete else 'trajectories/s'
    value = units / dt
    what = ('%d of the %d poses per step' if discrete else '%d of the %d trajectories per step') % (
        units, len(q) if discrete else len(off) - 1)
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': unit, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': dt * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': cfg['workload'], 'detector': cfg['kind'],
                       'reference': 'CPU restatement of the reference path (FP64 oracle, flags only); the upstream '
                                    'OptiX path is unavailable on this box (no RT cores, no OptiX SDK)'},
            'cpu_baseline': {'value': value, 'unit': unit, 'cores': threads, 'kind': 'port', 'sample': what},
            'e2e': {'value': value, 'unit': unit, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def _free_port():
    import socket
    sk = socket.socket()
    sk.bind(('127.0.0.1', 0))
    port = sk.getsockname()[1]
    sk.close()
    return port


def spawn_ranks(n):
    """`--gpus N` without an outside launcher: start N copies of this script,
    one per GPU, with RANK / LOCAL_RANK / WORLD_SIZE and a rendezvous on
    127.0.0.1 (what torch.distributed.run would set), and wait for them.
    Rank 0 prints the JSON line; the exit code is the worst of the ranks'."""
    port = _free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:], env=env))
    rc = 0
    for p in procs:
        rc = max(rc, p.wait())
    return rc


def run_dry(args, cfg, rank, world):
    """The multi-rank plumbing without a GPU (gloo on CPU): every rank checks
    its own seeded batch with the CPU oracle, the flags are all-gathered as
    in the GPU run, and rank 0 checks the gathered array against its own
    single-process run of every rank's batch."""
    import datetime

    import torch.distributed as dist
    from oracle import oracle as O
    from rtcollisiondetection_b200 import scenes, sharding
    if world > 1:
        dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        n = min(cfg['n'], args.dry_units)
        model, mesh, spheres, q, off = make_inputs(dict(cfg, n=n), rank, scenes)
        robot, scene = O.Robot(model, spheres=spheres), O.Scene(mesh)

        def check(q, off):
            if off is None:
                kind = O.ROBOT_TO_OBS if cfg['kind'] == 'RobotToObs' else O.OBS_TO_ROBOT
                return O.discrete(kind, robot, scene, q)['hit']
            return O.sweep(cfg['kind'] == 'Quadratic', robot, scene, q, off)['traj_hit']

        t0 = time.perf_counter()
        local = check(q, off)
        dt = sharding.max_over_ranks(time.perf_counter() - t0)
        flags = sharding.gather_flags(local, n * world, world)
        if rank == 0:
            want = np.concatenate([check(*make_inputs(dict(cfg, n=n), r, scenes)[3:]) for r in range(world)])
            line = {'metric': METRIC, 'value': n * world / dt, 'unit': 'trajectories/s' if off is not None else 'poses/s',
                    'n_gpus': world, 'steps': 1, 'warmup': 0, 'ms_per_step': dt * 1e3, 'higher_is_better': True,
                    'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                    'dry': 'CPU oracle per rank over gloo: exercises the launcher and the flag all-gather only',
                    'config': {'workload': cfg['workload'], 'units_per_gpu': n},
                    'gathered': {'units': int(len(flags)), 'equal_to_single_process': bool(np.array_equal(flags, want))}}
            print(json.dumps(line), flush=True)
            if not np.array_equal(flags, want):
                sys.exit(3)
    finally:
        if world > 1:
            dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--config', default='c2', choices=sorted(CONFIGS))
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-check', action='store_true')
    ap.add_argument('--ref-sample', type=int, default=8192)
    ap.add_argument('--plain-frame', type=int, default=1024, help='poses per frame of the plain arm (upstream batchSize)')
    ap.add_argument('--plain-streams', type=int, default=4, help='streams / host threads of the plain arm (upstream NSTREAM)')
    ap.add_argument('--fused', action='store_true', help='discrete: the thread-per-item traversal kernel')
    ap.add_argument('--no-graph', action='store_true', help='launch the timed steps directly, not as a CUDA graph')
    ap.add_argument('--two-way', action='store_true', help='discrete: both directions in one check (flags = union)')
    ap.add_argument('--containment', action='store_true', help='discrete: add the containment test')
    ap.add_argument('--serve-seconds', type=float, default=60.0,
                    help='length of the served mixed stream reported under "served" (0: skip)')
    ap.add_argument('--saturate-requests', type=int, default=4000,
                    help='requests of the served mix submitted at once to measure saturated throughput (0: skip)')
    ap.add_argument('--dry', action='store_true', help='no GPU: the multi-rank plumbing with the CPU oracle over gloo')
    ap.add_argument('--dry-units', type=int, default=256, help='units per rank of a --dry run')
    ap.add_argument('--units', type=int, default=0,
                    help='poses / trajectories per GPU instead of the configuration\'s (a smaller case for profiling)')
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.units:
        cfg['n'] = args.units
        cfg['workload'] += ' (%d units per GPU instead)' % args.units
    if args.gpus > 1 and 'WORLD_SIZE' not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if args.dry:
        run_dry(args, cfg, rank, world)
        return
    if args.impl == 'reference':
        run_reference(args, cfg, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120), device_id=torch.device('cuda', local))
    from rtcollisiondetection_b200 import rtcd, scenes
    model, mesh, spheres, q, off = make_inputs(cfg, rank, scenes)
    ctx = rtcd.Context(local)
    robot = rtcd.Robot(ctx, model, spheres=spheres)
    scene = rtcd.Scene.from_mesh(ctx, mesh)
    det = rtcd.Detector(ctx, cfg['kind'], robot, scene, frame_size=args.plain_frame, plain_streams=args.plain_streams)
    sweep = det.sweep
    n = cfg['n']
    # a dedicated stream: the legacy default stream has handle 0, which the ABI
    # reads as "the detector's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    qd = torch.from_numpy(q).cuda()
    fd = torch.zeros(n, dtype=torch.uint8, device='cuda')
    # sweeps: per-trajectory and per-segment flags (segment = linear capsule / quadratic piece or end sphere)
    n_seg = int(rtcd.segment_offsets(det.kind, off, 0)[-1]) if sweep else 0
    segd = torch.zeros(max(n_seg, 1), dtype=torch.uint8, device='cuda') if sweep else None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')

    tuned = det.autotune(qd, n, off, stream=sp)   # untimed: picks the traversal launch shape
    mode_flags = 0 if sweep else ((rtcd.CHECK_TWO_WAY if args.two_way else 0) |
                                  (rtcd.CHECK_CONTAINMENT if args.containment else 0))
    base_flags = rtcd.CHECK_TIMING | (rtcd.CHECK_FUSED if args.fused else 0) | mode_flags
    # the timed steps replay the launch sequence as a CUDA graph (captured in the first warm-up step)
    graph = 0 if args.no_graph else rtcd.CHECK_GRAPH

    def step(extra=0):
        det.check_device(qd, n, fd, traj_off=off, seg_dev=segd, flags=base_flags | extra, stream=sp)

    for _ in range(max(3, args.warmup)):
        step(graph)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    trav = []
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push('rtcd_timed')     # lets ncu restrict a launch list to the timed steps
    for k in range(args.steps):
        flush.fill_(k & 255)
        ev[k][0].record(stream)
        step(graph)
        ev[k][1].record(stream)
        trav.append(det.stats())   # syncs the step; the kernels' work counters of this step
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(np.sum(ms))
    if dist:
        t = torch.tensor([total_ms], device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / args.steps
    units_all = n * world
    value = units_all / (ms_step / 1e3)
    unit = 'trajectories/s' if sweep else 'poses/s'
    flags = fd.cpu().numpy()
    st = det.stats()
    gathered = None
    if dist:
        # the one exchange of the sharded path: every rank's flags, concatenated (NCCL all-gather);
        # rank 0 checks them against its own run of every rank's batch
        from rtcollisiondetection_b200 import sharding
        allf = sharding.gather_flags(flags, n * world, world, device=torch.device('cuda', local))
        if rank == 0:
            ok = True
            for r in range(world):
                qr, offr = make_inputs(cfg, r, scenes)[3:]
                ok &= bool(np.array_equal(det.check(qr, offr, flags=mode_flags)['flags'], allf[r * n:(r + 1) * n]))
            gathered = {'units': int(len(allf)), 'equal_to_rank0_rerun': ok}

    # end to end through the C ABI with host buffers (upload + download inside the call, in the graph):
    # the step's inputs arrive in pinned host memory, which the upload reads by DMA directly
    q_host = torch.empty(q.shape, dtype=torch.float32).pin_memory().numpy()
    q_host[...] = q
    e2e_ms = []
    for k in range(max(3, args.steps // 2) + 2):
        flush.fill_(k & 255)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = det.check(q_host, off, segments=sweep, flags=mode_flags | graph)
        dt = (time.perf_counter() - t0) * 1e3
        if k >= 2:
            e2e_ms.append(dt)
    e2e_step = float(np.mean(e2e_ms))
    assert np.array_equal(out['flags'], flags), 'host-buffer path disagrees with the device path'
    if sweep:
        assert np.array_equal(out['seg_flags'], segd.cpu().numpy()[:n_seg]), 'segment flags disagree'
    h2d = q.nbytes + (0 if off is None else off.nbytes)
    d2h = n + n_seg

    # plain path: the upstream check() shape - frames of 1,024 poses over 4 streams, one host thread per
    # stream, a host round trip per frame, a wait after every 4 frames; plus the 64-pose single-stream
    # frame path as a labelled extra
    plain = plain64 = None
    if not sweep:
        def time_plain(d):
            pm = []
            for k in range(3):
                flush.fill_(k & 255)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                d.check_device(qd, n, fd, flags=rtcd.CHECK_PLAIN | mode_flags, stream=sp)
                torch.cuda.synchronize()
                pm.append((time.perf_counter() - t0) * 1e3)
            assert np.array_equal(fd.cpu().numpy(), flags), 'plain path disagrees'
            return float(np.median(pm))
        pms = time_plain(det)
        plain = {'value': n / (pms / 1e3), 'unit': unit, 'frame': args.plain_frame, 'streams': args.plain_streams,
                 'host_threads': args.plain_streams, 'ms_per_step': pms,
                 'shape': 'upstream check(): frames round-robin over streams, one host thread per stream, item '
                          'count read back per frame, wait after every group of frames'}
        det64 = rtcd.Detector(ctx, cfg['kind'], robot, scene, frame_size=64, plain_streams=1)
        pm64 = time_plain(det64)
        det64.close()
        plain64 = {'value': n / (pm64 / 1e3), 'unit': unit, 'frame': 64, 'streams': 1, 'ms_per_step': pm64}

    peaks, peak_src = load_peaks()
    # traversal span of the same step, timed with events around its kernels (graph replays are timed whole)
    spans = []
    for k in range(3):
        flush.fill_(k & 255)
        step()
        spans.append(det.stats())
    t_trav = float(np.mean([s['ms_traverse'] for s in spans]))
    # algorithmic bytes of one traversal span: poses in, flags out, the resident structures read once
    if sweep:
        bytes_alg = n * 4 + int(q.nbytes) + 32 * scene.n_edges * 3
    else:
        bytes_alg = n * (4 * model['cos_mask'].shape[0] + 1) + (64 + 48) * scene.n_tris + (64 + 32) * 35991
    achieved = bytes_alg / (t_trav / 1e3) / 1e9
    form = tuned.get('stage_b_form', 0)
    if sweep:
        span = ('k_sweep_traj' if st['path_flags'] & 1 else 'k_sweep') + ' + k_sweep_heavy x 2 (heavy, split)'
    elif form in (0, 3, 4):
        span = 'k_stage_ab + k_subtree x 2 + k_stage_b (deferred) + k_stage_b_heavy + k_discrete (overflow)'
    else:
        span = 'k_stage_a + k_stage_b%s + k_stage_b_heavy + k_discrete (overflow)' % ('_packet' if form == 2 else '')
    traffic = None
    tp = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(tp):
        t = json.load(open(tp)).get(args.config)
        if t and t.get('span') == span:
            traffic = t['bytes_per_span']
    # FP32 work each kernel did, from its own counters, over its own event-timed duration (the
    # counters are the means over the timed steps; the durations the means over the span runs)
    links = model['cos_mask'].shape[0] + 1

    def mean(key, runs=trav):
        return float(np.mean([r[key] for r in runs]))

    nodes, leaves = mean('node_tests'), mean('exact_tests')
    nodes1, leaves1 = mean('first_node_tests'), mean('first_exact_tests')
    w_leaf = 40 if not sweep else (200 if cfg['kind'] == 'Quadratic' else 45)
    w_span = 18 * nodes + w_leaf * leaves
    w_first = 18 * nodes1 + w_leaf * leaves1
    if not sweep:
        cands = mean('candidates')
        w_span += 36 * cands   # every candidate primitive is moved into its link's frame
    t_first = float(np.mean([r['ms_first_pass'] for r in spans]))
    t_rest = max(t_trav - t_first, 1e-6)

    def kern(flops, ms):
        return {'flops': flops, 'ms': ms, 'achieved': flops / (ms / 1e3) / 1e12,
                'frac': flops / (ms / 1e3) / 1e12 / FP32_PEAK_TFLOPS}
    kernels = {'traversal_span': kern(w_span, t_trav),
               'first_pass': dict(kern(w_first, t_first), kernel=span.split(' + ')[0] + ' (light pass)' if sweep else
                                  ('k_stage_ab' if form in (0, 3, 4) else 'k_stage_a')),
               'later_passes': dict(kern(max(w_span - w_first, 0.0), t_rest),
                                    kernel='k_sweep_heavy' if sweep else
                                    'k_subtree x 2 + k_stage_b + k_stage_b_heavy + k_discrete')}
    if not sweep:
        sats, sph = mean('cull_sat_tests'), mean('cull_sphere_tests')
        t_cull = float(np.mean([r['ms_cull'] for r in spans]))
        kernels['cull'] = dict(kern(180 * sats + 8 * sph + 36 * n * (links - 1), t_cull),
                               kernel='k_cull + k_select_u8', sat_pairs=sats, sphere_tests=sph,
                               all_pairs=n * (links - 1) * scene.n_obstacles)
    fp32 = {'achieved': kernels['traversal_span']['achieved'], 'peak': FP32_PEAK_TFLOPS, 'unit': 'TFLOP/s',
            'frac': kernels['traversal_span']['frac'], 'flops_per_step': w_span,
            'node_tests': nodes, 'leaf_tests': leaves, 'kernels': kernels,
            'peak_source': 'nominal fallback: no FP32 peak in MEASURED_PEAKS.json '
                           '(148 SMs x 128 lanes x 2 x 1.965 GHz)',
            'weights': 'flops per counted op: node slab/box test 18, segment-triangle 40, segment-capsule 45, '
                       'segment-quadratic 200, candidate moved to the link frame 36, OBB SAT 180, '
                       'bounding-sphere test 8, world OBB 36'}
    if not args.no_check:
        fp32['reference_work'] = fp32_work(cfg, model, mesh, spheres, q, off, scene, t_trav)
    line = {
        'metric': METRIC, 'value': value, 'unit': unit, 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms_step, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic',
        'config': {'workload': cfg['workload'] + (' (two-way: both directions)' if args.two_way and not sweep else '')
                   + (' + containment' if args.containment and not sweep else ''),
                   'detector': cfg['kind'], 'units_per_gpu': n,
                   'l2': 'flushed before every step (256 MiB write)',
                   'form': 'batched: persistent traversal kernels, each step replayed as one CUDA graph'
                   if not args.no_graph else 'batched: persistent traversal kernels, launched directly',
                   'launch_shape': tuned},
        'e2e': {'value': units_all / (e2e_step / 1e3), 'unit': unit, 'ms_per_step': e2e_step,
                'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': int(d2h)},
        # discrete: k_fk_poses, k_cull, k_select_u8, then per direction k_stage_ab + k_subtree x 2 + k_stage_b
        # (deferred candidates) or k_stage_a + k_stage_b, k_stage_b_heavy, k_discrete (overflow); (k_contain),
        # k_flags; sweeps: k_fk_spheres, (k_fit), k_sweep, k_sweep_heavy, k_flags x 2
        # sweeps, staged light pass: k_sweep_traj, k_sweep_heavy, k_flags x 2; unstaged: k_fk_spheres, (k_fit),
        # k_sweep, k_sweep_heavy, k_flags x 2
        'gpu_launches': args.steps * ((3 + (2 if args.two_way else 1) * (6 if form in (0, 3, 4) else 4)
                                       + (1 if args.containment else 0) + 1) if not sweep
                                      # sweeps: light pass, heavy pass, its split pass, two flag gathers (+ FK and fit unstaged)
                                      else 5 if st['path_flags'] & 1 else (6 if cfg['kind'] == 'Linear' else 7)),
        'stages_ms': {'prepare': float(np.mean([s['ms_prepare'] for s in spans])),
                      'cull': float(np.mean([s['ms_cull'] for s in spans])), 'traverse': t_trav},
        'roofline': {'bound': 'hbm', 'kernel': span, 'achieved': achieved,
                     'peak': peaks['hbm_gbs'], 'unit': 'GB/s', 'frac': achieved / peaks['hbm_gbs'],
                     'traffic': traffic, 'peak_source': peak_src, 'fp32': fp32,
                     'note': 'latency-bound tree traversal: HBM is not the binding resource; achieved = algorithmic '
                             'bytes / traversal span (CUDA events on the launching stream); traffic = ncu DRAM '
                             'read+write of the span\'s kernels (profiles/traffic.json)'},
        'clocks': clocks,
    }
    if sweep and rank == 0:
        # the reference's entering-ray semantics beside the solid ones, on the same batch
        sem = {}
        for name, f in (('solid', 0), ('solid_no_end_spheres', rtcd.CHECK_NO_ENDPOINTS), ('surface', rtcd.CHECK_SURFACE)):
            o = det.check(q, off, segments=True, flags=f)
            sem[name] = o
        sf, ss = sem['surface'], sem['solid_no_end_spheres']
        sm = []
        for k in range(3):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            det.check_device(qd, n, fd, traj_off=off, flags=rtcd.CHECK_SURFACE, stream=sp)
            torch.cuda.synchronize()
            sm.append((time.perf_counter() - t0) * 1e3)
        line['semantics'] = {
            'traj_hit_rate': {k: float(v['flags'].mean()) for k, v in sem.items()},
            'seg_hit_rate': {k: float(v['seg_flags'].mean()) for k, v in sem.items()},
            'traj_solid_only': int(((sem['solid']['flags'] != 0) & (sf['flags'] == 0)).sum()),
            'seg_solid_only': int(((ss['seg_flags'] != 0) & (sf['seg_flags'] == 0)).sum()),
            'seg_surface_only': int(((ss['seg_flags'] == 0) & (sf['seg_flags'] != 0)).sum()),
            'segments': int(len(sf['seg_flags'])),
            'surface_units_per_s': n / (np.median(sm) / 1e3),
            'note': 'solid: an obstacle edge within r of the sphere path (round caps; quadratic adds the start/end '
                    'spheres); surface: the reference semantics, a directed loop edge entering a piece (flat '
                    'quadratic caps, no end spheres); seg_* compare surface with solid without end spheres'}
        if not args.no_check:
            from oracle import oracle as O
            m = min(len(off) - 1, 128)
            ref = O.sweep(cfg['kind'] == 'Quadratic', O.Robot(model, spheres=spheres), O.Scene(mesh), q[:off[m]],
                          off[:m + 1], surface=True)
            line['semantics']['surface_check'] = {
                'flag_errors': int(((sf['flags'][:m] != ref['traj_hit']) & (ref['traj_band'] == 0)).sum()),
                'seg_flag_errors': int(((sf['seg_flags'][:ref['seg_off'][-1]] != ref['seg_hit'])
                                        & (ref['seg_band'] == 0)).sum()),
                'checked': m, 'in_band': int(ref['traj_band'].sum())}
    if gathered:
        line['gathered'] = gathered
    if plain:
        # per GPU on both sides: the plain arm runs on rank 0's GPU alone
        line['plain'] = plain
        line['batched_over_plain'] = value / world / plain['value']
        line['plain_frame64'] = plain64
        line['batched_over_plain_frame64'] = value / world / plain64['value']
    if not args.no_check and rank == 0:
        line['check'] = oracle_errors(cfg, model, mesh, spheres, q, off, flags, two_way=args.two_way,
                                      containment=args.containment)
        line['fp64_retests'] = st['fp64_retests']
        line['fp64'] = dict(fp64_statement(cfg, ctx, model, mesh, spheres, q, off),
                            retests_per_step=st['fp64_retests'],
                            root_findings_per_step=st['candidates'] if cfg['kind'] == 'Quadratic' else None,
                            in_band_of_checked=line['check']['in_band'])
    # the served stream is a one-GPU measurement: a scaling run (N > 1) skips it
    if args.serve_seconds > 0 and rank == 0 and world == 1 and args.config == 'c2':
        line['served'] = served_stream(ctx, args.serve_seconds, saturate_requests=args.saturate_requests)
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        line['cpu_baseline'] = cpu_baseline(cfg, model, mesh, spheres, q, off)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del det, scene, robot, ctx
    if dist:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
