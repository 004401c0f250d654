"""The benchmark's reference arm (`bench.py --impl reference`) runs on the host alone
and prints one JSON line with the contract's keys: the numpy oracle timed on a
bounded sample of the benchmark workload, with its e2e equal to its value."""
import json
import os
import subprocess
import sys

from .conftest import ROOT


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--steps', '1',
                          '--warmup', '1', '--batch', '32'], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith('{')][-1])
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better',
                'scaling', 'vs_baseline', 'dtype', 'data', 'config', 'impl', 'cpu_baseline', 'e2e'):
        assert key in line, key
    assert line['impl'] == 'reference' and line['value'] > 0 and line['higher_is_better'] is True
    assert line['cpu_baseline']['kind'] == 'port' and line['cpu_baseline']['cores'] >= 1
    assert line['e2e']['value'] == line['value'] and line['e2e']['h2d_bytes_per_step'] == 0
    assert line['config']['workload'].startswith('multislice LSQ-ML')
    # the same config keys as the GPU arm's line (single GPU)
    assert line['config']['parallelism'] == 'single GPU'
    assert '32 positions' in line['cpu_baseline']['sample']
