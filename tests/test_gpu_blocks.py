"""Building blocks on the device: FK, scan, compaction, LBVH - each against
the oracle or a plain CPU restatement of the same operation."""
import numpy as np
import pytest

from oracle import oracle as O
from rtcollisiondetection_b200 import rtcd, scenes

pytestmark = pytest.mark.gpu


def test_fk_matches_fp64(ctx, panda):
    import torch
    robot = rtcd.Robot(ctx, panda)
    q = scenes.uniform_poses(panda, 4096, seed=3)
    # include the joint limits themselves
    q[:2] = np.stack([panda['lower'], panda['upper']])
    qd = torch.from_numpy(q).cuda()
    T = torch.zeros((len(q), 8, 12), dtype=torch.float32, device='cuda')
    rtcd.robot_fk(robot, qd, len(q), T)
    torch.cuda.synchronize()
    ref = O.fk(panda, q)
    err = np.abs(T.cpu().numpy().astype(np.float64) - ref)
    # link origins (translation column) within 1e-5 m of FP64, rotations within 1e-5
    assert err[..., [3, 7, 11]].max() < 1e-5
    assert err.max() < 1e-5


@pytest.mark.parametrize('n', [0, 1, 4, 2047, 2048, 2049, 4096, 8192, 41616, 1 << 20])
def test_exclusive_scan_known_answer(ctx, n):
    """Sizes straddle the 2048-element tile (upstream testExclusiveScan.cpp:27-80
    checks against std::exclusive_scan)."""
    import torch
    rng = np.random.default_rng(n)
    x = rng.integers(0, 1000, size=n, dtype=np.uint32)
    xi = torch.from_numpy(x.astype(np.int32)).cuda()
    out = torch.zeros(max(n, 1), dtype=torch.int32, device='cuda')
    total = torch.zeros(1, dtype=torch.int32, device='cuda')
    rtcd.exclusive_scan_u32(ctx, xi, out, n, total)
    torch.cuda.synchronize()
    ref = np.concatenate([[0], np.cumsum(x, dtype=np.uint64)[:-1]]).astype(np.uint32) if n else np.zeros(0, np.uint32)
    assert np.array_equal(out.cpu().numpy()[:n].astype(np.uint32), ref)
    assert int(total.item()) == int(x.sum())


@pytest.mark.parametrize('n,p', [(0, 0.5), (1, 1.0), (2048, 0.3), (4097, 0.5), (100000, 0.01), (1 << 20, 0.7)])
def test_select_known_answer(ctx, n, p):
    """Stable compaction against a CPU filter (upstream testStreamCompact.cpp:27-101)."""
    import torch
    rng = np.random.default_rng(n + 7)
    m = (rng.random(n) < p).astype(np.uint8)
    md = torch.from_numpy(m).cuda()
    idx = torch.zeros(max(n, 1), dtype=torch.int32, device='cuda')
    cnt = torch.zeros(1, dtype=torch.int32, device='cuda')
    rtcd.select_flags_u8(ctx, md, n, idx, cnt)
    torch.cuda.synchronize()
    ref = np.nonzero(m)[0]
    assert int(cnt.item()) == len(ref)
    assert np.array_equal(idx.cpu().numpy()[:len(ref)], ref)


@pytest.mark.parametrize('which', ['small_tris', 'small_edges', 'dense_tris', 'dense3_tris', 'dense3_edges', 'one', 'two',
                                   'dupes'])
def test_lbvh_bit_identical_to_canonical(ctx, which):
    if which in ('small_tris', 'small_edges', 'dense_tris', 'dense3_tris', 'dense3_edges'):
        m = {'dense_tris': lambda: scenes.discrete_dense(ico_level=2), 'dense3_tris': scenes.discrete_dense,
             'dense3_edges': scenes.discrete_dense}.get(which, scenes.discrete_small)()
        v = m.verts.astype(np.float32)
        if which in ('small_edges', 'dense3_edges'):
            e = O.unique_edges(m.tris)
            P = v[e]
        else:
            P = v[m.tris]
        lo, hi = P.min(1), P.max(1)
    elif which == 'one':
        lo, hi = np.zeros((1, 3), np.float32), np.ones((1, 3), np.float32)
    elif which == 'two':
        lo = np.array([[0, 0, 0], [1, 1, 1]], np.float32)
        hi = lo + 0.5
    else:  # many identical boxes: equal Morton codes, index tie-breaks
        lo = np.repeat(np.array([[0.5, 0.5, 0.5]], np.float32), 300, 0)
        lo[::7] += 0.25
        hi = lo + 0.01
    g = rtcd.lbvh_build(ctx, lo, hi)
    codes, perm, child, nlo, nhi = O.lbvh(lo, hi)
    assert np.array_equal(g['codes'], codes)
    assert np.array_equal(g['perm'], perm)
    n = len(lo)
    if n > 1:
        # oracle children: >=0 internal, <0 leaf ~s; device: bit31 leaf
        dev = g['child'].astype(np.int64)
        conv = np.where(dev & 0x80000000, ~(dev & 0x7fffffff), dev)
        assert np.array_equal(conv, child.astype(np.int64))
        assert np.array_equal(g['node_lo'], nlo) and np.array_equal(g['node_hi'], nhi)
    assert g['depth'] <= 62


@pytest.mark.parametrize('n', [1, 5000, 70001])
def test_lookback_wait_runs_out_and_reports(ctx, n):
    """Failure detection of the bounded device waits, made to fire on purpose:
    tile 0 of the look-back compaction never publishes (no block takes it),
    so every other tile's wait runs out after a short spin limit.  The kernel
    must return, the call must report RTCD_ERR_DEVICE_TIMEOUT, and the context
    must stay usable: a normal compaction on it afterwards is exact."""
    import time

    import torch
    t0 = time.time()
    st = rtcd.selftest_lookback_timeout(ctx, n, 256)
    assert st == 4, (st, rtcd.last_error())  # RTCD_ERR_DEVICE_TIMEOUT
    assert 'ran out' in rtcd.last_error()
    assert time.time() - t0 < 30.0
    m = (np.arange(4097) % 3 == 0).astype(np.uint8)
    md = torch.from_numpy(m).cuda()
    idx = torch.zeros(len(m), dtype=torch.int32, device='cuda')
    cnt = torch.zeros(1, dtype=torch.int32, device='cuda')
    rtcd.select_flags_u8(ctx, md, len(m), idx, cnt)
    torch.cuda.synchronize()
    ref = np.nonzero(m)[0]
    assert int(cnt.item()) == len(ref)
    assert np.array_equal(idx.cpu().numpy()[:len(ref)], ref)
