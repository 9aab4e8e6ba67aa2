"""bench.py's reference arm (the CPU oracle timed on the host) prints the one
JSON line the measurement contract asks for, with its e2e and cpu_baseline
objects; it needs no GPU, so it runs here on the small configuration."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), *args], capture_output=True, text=True,
                         cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith('{')]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run_bench('--impl', 'reference', '--config', 'c1', '--steps', '1', '--warmup', '3')
    for k in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'scaling',
              'vs_baseline', 'dtype', 'data', 'config', 'e2e', 'cpu_baseline'):
        assert k in d, k
    assert d['impl'] == 'reference' and d['n_gpus'] == 1 and d['steps'] == 1 and d['warmup'] == 3
    assert d['value'] > 0 and d['unit'] == 'poses/s' and d['higher_is_better'] is True
    assert d['e2e']['value'] == d['value'] and d['e2e']['h2d_bytes_per_step'] == 0
    cb = d['cpu_baseline']
    assert cb['value'] == d['value'] and cb['kind'] in ('port', 'reference') and cb['cores'] >= 1
    assert d['config']['workload']


def test_two_rank_launcher_gathers_flags_on_cpu():
    """`bench.py --gpus 2` starts two ranks itself (RANK / LOCAL_RANK /
    WORLD_SIZE, rendezvous on 127.0.0.1); the --dry path runs them over gloo
    with the CPU oracle, all-gathers the flags and rank 0 checks the gathered
    array against a single-process run of both ranks' batches."""
    d = run_bench('--gpus', '2', '--dry', '--config', 'c1', '--dry-units', '128')
    assert d['n_gpus'] == 2 and d['scaling'] == 'weak'
    assert d['gathered'] == {'units': 256, 'equal_to_single_process': True}


def test_two_rank_launcher_sweep_on_cpu():
    d = run_bench('--gpus', '2', '--dry', '--config', 'c3', '--dry-units', '16')
    assert d['n_gpus'] == 2 and d['unit'] == 'trajectories/s'
    assert d['gathered'] == {'units': 32, 'equal_to_single_process': True}
