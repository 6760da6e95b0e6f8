"""The multi-rank host logic of bench.py on CPU (gloo, world size 2): the
job time is the maximum over ranks, and under torchrun the reference arm
runs on rank 0 only.  The collectives of the frame-sharded iteration itself
are tested in test_shard.py (CPU) and test_gpu_shard.py."""
import os
import socket
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import datetime, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))
rank = dist.get_rank()
v = bench.max_over_ranks(1.5 + 2.0 * rank, 'cpu')
dist.barrier()
dist.destroy_process_group()
print('rank %d max %r' % (rank, v))
'''


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_max_over_ranks_gloo(tmp_path):
    script = tmp_path / 'worker.py'
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE='2', LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, str(script), REPO], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err
    got = sorted(o.strip() for o, _ in outs)
    assert got == ['rank 0 max 3.5', 'rank 1 max 3.5']


def test_max_over_ranks_single_process():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(2.25, 'cpu') == 2.25


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 times the reference; rank 1 prints nothing
    and exits 0 at once."""
    env = dict(os.environ, RANK='1', WORLD_SIZE='2', LOCAL_RANK='1')
    r = subprocess.run([sys.executable, os.path.join(REPO, 'bench.py'), '--impl', 'reference',
                        '--gpus', '2'], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ''
