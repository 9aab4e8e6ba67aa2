"""The C++ facade (include/rtcd/CollisionDetector.hpp) with the upstream call
sequence: compiled and linked on any host, run on the GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, 'rtcollisiondetection_b200')


def _build(tmp_path):
    from rtcollisiondetection_b200 import rtcd
    rtcd.lib()  # the engine must exist
    exe = str(tmp_path / 'facade_check')
    cxx = shutil.which('g++') or shutil.which('c++')
    subprocess.check_call([cxx, '-std=c++17', '-Wall', '-Werror', '-I', os.path.join(ROOT, 'include'),
                           os.path.join(ROOT, 'tests', 'cpp', 'facade_check.cpp'), '-L', LIBDIR, '-lrtcd_b200',
                           '-Wl,-rpath,' + LIBDIR, '-o', exe])
    return exe


def test_facade_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_facade_runs_upstream_sequence(tmp_path):
    out = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = dict(l.split(':', 1) for l in out.stdout.strip().splitlines())
    assert lines['flags'].split() == ['1', '0']
    assert lines['counts'].split() == ['3', '0']
