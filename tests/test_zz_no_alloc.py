"""The allocation-free compaction entry point.

rtcd_select_flags_u8_noalloc serves callers that cannot allocate device
memory when they query (hard-deadline control loops, processes whose device
memory belongs to another owner): its look-back scratch is a fixed array
inside the library.  This test calls it through the C ABI and checks that it
returns exactly what the allocating entry point rtcd_select_flags_u8 returns
(indices are integers: the comparison is exact), on two calls in a row whose
sizes differ so the second call must not see the first call's scratch.  This
file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from rtcollisiondetection_b200 import rtcd

pytestmark = pytest.mark.gpu


def _noalloc(mask_dev, n, idx_dev, cnt_dev, stream):
    lib = rtcd.lib()
    fn = lib.rtcd_select_flags_u8_noalloc
    fn.restype = C.c_int
    return fn(C.c_void_p(mask_dev.data_ptr()), C.c_uint32(n), C.c_void_p(idx_dev.data_ptr()),
              C.c_void_p(cnt_dev.data_ptr()), C.c_void_p(stream))


def test_noalloc_select_matches_allocating_entry_point():
    import torch
    ctx = rtcd.Context(0)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for call, (n, p, seed) in enumerate([(3_000_001, 0.37, 1), (70_001, 0.9, 2)]):
            rng = np.random.default_rng(seed)
            m = (rng.random(n) < p).astype(np.uint8)
            md = torch.from_numpy(m).cuda()
            idx_a = torch.full((n,), -1, dtype=torch.int32, device='cuda')
            idx_b = torch.full((n,), -1, dtype=torch.int32, device='cuda')
            cnt_a = torch.zeros(1, dtype=torch.int32, device='cuda')
            cnt_b = torch.full((1,), -1, dtype=torch.int32, device='cuda')
            s.synchronize()
            rtcd.select_flags_u8(ctx, md, n, idx_a, cnt_a, stream=s.cuda_stream)
            st = _noalloc(md, n, idx_b, cnt_b, s.cuda_stream)
            assert st == 0, rtcd.last_error()
            s.synchronize()
            k = int(cnt_a.item())
            assert k == int(m.sum()), call
            assert int(cnt_b.item()) == k, call
            assert torch.equal(idx_a[:k], idx_b[:k]), call
    ctx.close()


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch
    buf = torch.zeros(16, dtype=torch.int32, device='cuda')
    st = _noalloc(buf, (1 << 25) + 1, buf, buf, 0)
    assert st == 5  # RTCD_ERR_CAPACITY, raised before any device work
    assert '33554432' in rtcd.last_error()
