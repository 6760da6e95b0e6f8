"""Host logic of the frame-sharded multi-GPU EMC (rspi/shard.py) on CPU with
two gloo ranks: frame and pixel blocks, the dataset-wide statistics from
exact integer sums (bit-identical to one process), the histogram sum, the
gather of each rank's pattern-search pixels and of per-frame argmaxes."""
import os
import socket
import subprocess
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, 'refspi-maxlp_b200'))


def test_block_range_partitions():
    from rspi.shard import block_range
    for n in (0, 1, 7, 100, 20001):
        for size in (1, 2, 3, 8):
            blocks = [block_range(n, r, size) for r in range(size)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            assert max(b - a for a, b in blocks) - min(b - a for a, b in blocks) <= 1


def test_frames_of_host_concatenate_back():
    from helpers import random_photons
    from rspi.shard import block_range, frames_of_host
    d = random_photons(17, 23, 300., 5, empty_frames=(3,))
    host = dict(num_data=23, ones=d['ones'], multi=d['multi'], place_ones=d['place_ones'],
                place_multi=d['place_multi'], count_multi=d['count_multi'])
    parts = [frames_of_host(host, *block_range(23, r, 3)) for r in range(3)]
    for key in ('ones', 'multi', 'place_ones', 'place_multi', 'count_multi'):
        assert np.array_equal(np.concatenate([p[key] for p in parts]), host[key]), key
    assert sum(p['num_data'] for p in parts) == 23


WORKER = r'''
import datetime, os, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch
import torch.distributed as dist
from rspi import shard
dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))
rank, size = shard.world()
rng = np.random.default_rng(0)
n, npix = 11, 50
counts = rng.integers(0, 400, n)
sums = rng.integers(0, 30, (n, npix)).astype('f8')
lo, hi = shard.block_range(n, rank, size)
# statistics of the whole dataset from this rank's exact sums
photons = int(counts[lo:hi].sum())
n_all, mc, scales, powder = shard.combine_stats(
    photons, hi - lo, torch.from_numpy(sums[lo:hi].sum(0)),
    torch.from_numpy(counts[lo:hi]), True)
mc1 = float(counts.sum()) / float(n)
assert n_all == n and mc == mc1
assert np.array_equal(scales.numpy(), counts[lo:hi].astype('f8') / mc1)
assert np.array_equal(powder.numpy(), sums.sum(0) / float(n))
# histogram: integer sums over ranks
hist = torch.full((6,), rank + 1, dtype=torch.int32)
nstate = torch.full((3,), 2 * rank, dtype=torch.int32)
class Stub:
    size = 4
    main = torch.tensor([1, 2, 5, 6, 9, 10, 13], dtype=torch.int32)
    n_main = 7
sm = shard.ShardedMStep(Stub())
sm.reduce_histogram(hist, nstate)
assert hist.tolist() == [3] * 6 and nstate.tolist() == [2] * 3
# each rank updates its block of the main pixels; the gather gives all
model0 = torch.from_numpy(rng.random(16) + 1j * rng.random(16))
f = model0.clone()
mlo, mhi = sm.main_block()
mine = Stub.main[mlo:mhi]
f[mine.long()] = -(1 + rank) * (1 + 1j) * f[mine.long()]
sm.gather_main(f, mine)
want = model0.clone()
for r in range(size):
    a, b = shard.block_range(7, r, size)
    idx = Stub.main[a:b].long()
    want[idx] = -(1 + r) * (1 + 1j) * model0[idx]
assert torch.equal(f, want)
# per-frame argmaxes in frame order
rm = torch.arange(lo, hi, dtype=torch.int32) * 10
assert torch.equal(shard.gather_frames(rm, n), torch.arange(n, dtype=torch.int32) * 10)
dist.barrier()
dist.destroy_process_group()
print('rank %d ok' % rank)
'''


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_shard_collectives_gloo(tmp_path):
    script = tmp_path / 'worker.py'
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE='2', LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES='')
        procs.append(subprocess.Popen([sys.executable, str(script),
                                       os.path.join(REPO, 'refspi-maxlp_b200')], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    outs = [p.communicate(timeout=120)[0].decode() for p in procs]
    for rank, (p, out) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, out
        assert 'rank %d ok' % rank in out
