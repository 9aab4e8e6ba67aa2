"""Planner side: neighbour search against numpy, and batched straight-line
edge checks against the same edges built on the host and checked with
rtcd_check (sweeps: one trajectory per edge; discrete: every configuration)."""
import numpy as np
import pytest
import torch

from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


def _numpy_knn(p, k, w, mask=None):
    d2 = (((p[:, None, :] - p[None, :, :]) * w) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    if mask is not None:
        d2[mask, :] = np.inf
        d2[:, mask] = np.inf
    order = np.argsort(d2, axis=1, kind='stable')[:, :k]
    return order, np.sqrt(np.take_along_axis(d2, order, 1)), d2


@pytest.mark.parametrize('n,k', [(1000, 10), (257, 32), (40, 1)])
def test_knn_matches_numpy(ctx, panda, n, k):
    pts = rtcd.halton_samples(n, panda['lower'], panda['upper'])
    w = np.linspace(1.0, 0.4, 7).astype(np.float32)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        pd = torch.from_numpy(pts).cuda()
        idx = torch.zeros((n, k), dtype=torch.int32, device='cuda')
        dist = torch.zeros((n, k), dtype=torch.float32, device='cuda')
        rtcd.knn(ctx, pd, n, 7, k, idx, dist, weights=w, stream=s.cuda_stream)
        s.synchronize()
    gi, gd = idx.cpu().numpy().view(np.uint32), dist.cpu().numpy()
    ri, rd, d2 = _numpy_knn(pts.astype(np.float64), k, w.astype(np.float64))
    assert np.allclose(gd, rd, rtol=2e-5, atol=1e-6)
    # indices agree except where neighbouring distances tie within float rounding
    srt = np.sort(d2, axis=1)
    sharp = np.all(np.diff(srt[:, :k + 1], axis=1) > 1e-5 * srt[:, 1:k + 1], axis=1)
    assert sharp.mean() > 0.9
    assert np.array_equal(gi[sharp], ri[sharp])


def test_knn_mask_and_short_rows(ctx, panda):
    n, k = 50, 8
    pts = rtcd.halton_samples(n, panda['lower'], panda['upper'], skip=3)
    mask = np.zeros(n, np.uint8)
    mask[::2] = 1
    mask[1:45:2] = 1           # 3 points left: each has 2 neighbours
    pd = torch.from_numpy(pts).cuda()
    md = torch.from_numpy(mask).cuda()
    idx = torch.zeros((n, k), dtype=torch.int32, device='cuda')
    dist = torch.zeros((n, k), dtype=torch.float32, device='cuda')
    rtcd.knn(ctx, pd, n, 7, k, idx, dist, mask_dev=md)
    torch.cuda.synchronize()
    gi, gd = idx.cpu().numpy().view(np.uint32), dist.cpu().numpy()
    free = np.nonzero(mask == 0)[0]
    assert len(free) == 3
    for q in free:
        assert set(gi[q, :2]) == set(free) - {q}
        assert (gi[q, 2:] == 0xFFFFFFFF).all() and (gd[q, 2:] == np.finfo(np.float32).max).all()
    assert (gi[mask == 1] == 0xFFFFFFFF).all()


def _host_edges(nodes, edges, n_wp):
    a, b = nodes[edges[:, 0]], nodes[edges[:, 1]]
    span = (b - a) / np.float32(n_wp - 1)
    i = np.arange(n_wp, dtype=np.float32)[None, :, None]
    return (a[:, None, :] + span[:, None, :] * i).astype(np.float32).reshape(-1, nodes.shape[1])


@pytest.mark.parametrize('kind,n_wp', [('Linear', 12), ('Quadratic', 9), ('RobotToObs', 10), ('ObsToRobot', 6)])
def test_edge_checks_match_host_built_edges(ctx, panda, small_scene, kind, n_wp):
    """A PRM-style roadmap: Halton samples, k nearest neighbours on the GPU,
    every (sample, neighbour) edge checked in one call."""
    n, k = 300, 6
    nodes = rtcd.halton_samples(n, panda['lower'], panda['upper'])
    sph = scenes.synth_spheres(panda)
    robot = rtcd.Robot(ctx, panda, spheres=sph)
    sc = rtcd.Scene.from_mesh(ctx, small_scene)
    det = rtcd.Detector(ctx, kind, robot, sc)
    nd = torch.from_numpy(nodes).cuda()
    idx = torch.zeros((n, k), dtype=torch.int32, device='cuda')
    dist = torch.zeros((n, k), dtype=torch.float32, device='cuda')
    rtcd.knn(ctx, nd, n, 7, k, idx, dist)
    torch.cuda.synchronize()
    nb = idx.cpu().numpy().view(np.uint32)
    edges = np.stack([np.repeat(np.arange(n, dtype=np.uint32), k), nb.reshape(-1)], axis=1)
    m = len(edges)
    ed = torch.from_numpy(edges.astype(np.int32)).cuda()
    fd = torch.zeros(m, dtype=torch.uint8, device='cuda')
    det.check_edges(nd, n, ed, m, n_wp, fd)
    torch.cuda.synchronize()
    got = fd.cpu().numpy()
    q = _host_edges(nodes, edges, n_wp)
    if det.sweep:
        off = (np.arange(m + 1) * n_wp).astype(np.uint32)
        ref = det.check(q, off)['flags']
    else:
        ref = det.check(q)['flags'].reshape(m, n_wp).max(axis=1)
    assert np.array_equal(got, ref)
    assert 0.05 < got.mean() < 0.95
    if not det.sweep:   # two-way over the same edges is the union of both directions
        fd2 = torch.zeros(m, dtype=torch.uint8, device='cuda')
        det.check_edges(nd, n, ed, m, n_wp, fd2, flags=rtcd.CHECK_TWO_WAY)
        other = rtcd.Detector(ctx, 'ObsToRobot' if kind == 'RobotToObs' else 'RobotToObs', robot, sc)
        ref2 = ref | other.check(q)['flags'].reshape(m, n_wp).max(axis=1)
        torch.cuda.synchronize()
        assert np.array_equal(fd2.cpu().numpy(), ref2)


def test_edge_check_rejects_bad_input(ctx, panda, small_scene):
    robot = rtcd.Robot(ctx, panda)
    det = rtcd.Detector(ctx, 'RobotToObs', robot, rtcd.Scene.from_mesh(ctx, small_scene))
    nd = torch.zeros((4, 7), device='cuda')
    ed = torch.zeros((2, 2), dtype=torch.int32, device='cuda')
    fd = torch.zeros(2, dtype=torch.uint8, device='cuda')
    with pytest.raises(rtcd.RTCDError):
        det.check_edges(nd, 4, ed, 2, 1, fd)                     # fewer than 2 configurations per edge
    with pytest.raises(rtcd.RTCDError):
        det.check_edges(nd, 4, ed, 2, 5, fd, flags=rtcd.CHECK_COUNTS)
