"""The N > 1 path of bench.py on CPU: two gloo ranks agree on the slowest
rank's step time, and the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


_WORKER = r'''
import os, sys, datetime
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
v = bench.max_over_ranks(1.5 + r, 'cpu')
dist.barrier()
dist.destroy_process_group()
print('RESULT', r, v)
'''


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE='2', LOCAL_RANK=str(r),
                   MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, '-c', _WORKER, ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(out)
    vals = sorted(float(line.split()[2]) for o in outs for line in o.splitlines()
                  if line.startswith('RESULT'))
    assert vals == [2.5, 2.5]


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK='1', WORLD_SIZE='2', LOCAL_RANK='1')
    p = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference'],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ''
