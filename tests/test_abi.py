"""The C-ABI library loads and exports every symbol include/rtcd.h declares
(no device calls)."""
import ctypes
import os
import re

from rtcollisiondetection_b200 import rtcd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, 'include', 'rtcd.h')).read()
    return sorted(set(re.findall(r'RTCD_API\s+[\w\s\*]+?\b(rtcd_\w+)\s*\(', src)))


def test_header_declares_the_abi():
    names = declared()
    for must in ('rtcd_context_create', 'rtcd_robot_create', 'rtcd_scene_create', 'rtcd_detector_create',
                 'rtcd_check', 'rtcd_sync', 'rtcd_last_error'):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = rtcd.lib()
    for name in declared():
        assert hasattr(lib, name), name
    assert set(rtcd.EXPORTS) <= set(declared())
    assert lib.rtcd_abi_version() == 1


def test_last_error_is_empty_and_bounded():
    buf = ctypes.create_string_buffer(4)
    assert rtcd.lib().rtcd_last_error(buf, ctypes.c_size_t(4)) == 0


def test_segment_offsets_host_only():
    """Pure host logic: segments per trajectory for both sweep kinds."""
    off = [0, 8, 17, 81, 84]
    lin = rtcd.segment_offsets(rtcd.LINEAR_SWEEP, off)
    assert lin.tolist() == [0, 7, 15, 78, 80]
    quad = rtcd.segment_offsets(rtcd.QUAD_SWEEP, off)
    # nc = max(3, ceil(n/2)): 4, 5, 32, 3 -> pieces nc - 2 + 2
    assert quad.tolist() == [0, 4, 9, 41, 44]
    quad_ne = rtcd.segment_offsets(rtcd.QUAD_SWEEP, off, rtcd.CHECK_NO_ENDPOINTS)
    assert quad_ne.tolist() == [0, 2, 5, 35, 36]
    try:
        rtcd.segment_offsets(rtcd.ROBOT_TO_OBS, off)
        assert False
    except rtcd.RTCDError as e:
        assert e.status == 1


def test_library_weight_fit_matches_shipped_tables():
    """Host-only: the library's banded least-squares fit reproduces every
    shipped RTCD/data/weights/quad/normal table (the golden fixtures)."""
    import numpy as np
    g = np.load(os.path.join(ROOT, 'tests', 'golden', 'quad_weights.npz'))
    for k in g.files:
        nc, nt = map(int, k[2:].split('_'))
        W = rtcd.quad_fit_weights(nc, nt)
        assert np.abs(W - g[k]).max() < 2e-6, k
    try:
        rtcd.quad_fit_weights(2, 8)
        assert False
    except rtcd.RTCDError as e:
        assert e.status == 1
