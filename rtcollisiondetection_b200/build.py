"""Builds the engine: every CUDA source under csrc/ is compiled for sm_100a by
nvcc and linked into ``librtcd_b200.so`` next to this file (in-tree, so the
library travels with the repository)."""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, 'librtcd_b200.so')
SOURCES = sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cu')))
HEADERS = sorted(glob.glob(os.path.join(HERE, 'csrc', '*.h')) + glob.glob(os.path.join(HERE, 'csrc', '*.cuh')) +
                 glob.glob(os.path.join(ROOT, 'include', '*.h')))
NVCC = os.environ.get('NVCC', 'nvcc')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC',
         '-Xcompiler', '-fvisibility=hidden', '-I' + os.path.join(ROOT, 'include')]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, '_build')
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.basename(src) + '.o')
        objs.append(obj)
        cmd = [NVCC] + FLAGS + ['-c', src, '-o', obj]
        if verbose:
            print(' '.join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for src, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode:
            raise RuntimeError('nvcc failed on %s:\n%s' % (src, out))
    cmd = [NVCC, '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', '-o', LIB + '.tmp'] + objs + ['-lcudart']
    subprocess.check_call(cmd)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True)
    print(LIB)
