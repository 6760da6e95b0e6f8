"""Frame-sharded EMC on the GPU: two ranks (processes on the one GPU of
this run, host-side gloo collectives; on a multi-GPU node the same code runs
one process per GPU over NCCL) give the single-process argmax and model bit
for bit, from one photons file split in frame blocks and from per-rank
files.  The ranks' kernels never wait on each other: every exchange is a
host collective between iterations' stages."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch

from helpers import load_golden, write_case

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import datetime, os, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch
import torch.distributed as dist
torch.cuda.set_device(0)
dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=120))
from emc import EMC
rec = EMC(sys.argv[2])
rec.model = np.load(sys.argv[3])
for it in (1, 2):
    rec.run_iteration(it)
    if dist.get_rank() == 0:
        np.save(sys.argv[4] + '_rmax%d.npy' % it, rec.rmax)
        np.save(sys.argv[4] + '_model%d.npy' % it, rec.model)
dist.barrier()
dist.destroy_process_group()
print('done')
'''


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _run_ranks(tmp_path, cfg, model_path, out_prefix, n=2):
    script = tmp_path / 'worker.py'
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for rank in range(n):
        env = dict(os.environ, MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE=str(n), LOCAL_RANK=str(rank), RSPI_AUTOTUNE_CACHE=str(
                       tmp_path / ('tune%d.json' % rank)))
        procs.append(subprocess.Popen(
            [sys.executable, str(script), os.path.join(REPO, 'refspi-maxlp_b200'), cfg,
             model_path, out_prefix], env=env, stdout=subprocess.PIPE,
            stderr=subprocess.STDOUT))
    outs = [p.communicate(timeout=600)[0].decode() for p in procs]
    for p, out in zip(procs, outs):
        assert p.returncode == 0, out[-3000:]


def _single(cfg, model):
    from emc import EMC
    rec = EMC(cfg)
    rec.model = model.copy()
    out = []
    for it in (1, 2):
        rec.run_iteration(it)
        out.append((rec.rmax.copy(), rec.model.copy()))
    return out


@pytest.mark.parametrize('pre_sharded', [False, True])
def test_two_ranks_equal_one(tmp_path, pre_sharded):
    from rspi.photonfile import write_photons
    from rspi.shard import block_range, frames_of_host
    g = load_golden('case_a')
    cfg = write_case(str(tmp_path), g=g)
    model = g['model_in_1'].copy()
    model_path = str(tmp_path / 'model0.npy')
    np.save(model_path, model)
    want = _single(cfg, model)
    if pre_sharded:
        # one file per rank: the frame blocks of the same data
        host = dict(num_data=int(g['ones'].size), ones=g['ones'], multi=g['multi'],
                    place_ones=g['place_ones'], place_multi=g['place_multi'],
                    count_multi=g['count_multi'])
        for r in range(2):
            part = frames_of_host(host, *block_range(host['num_data'], r, 2))
            part['num_pix'] = np.array([int(g['size']) ** 2])
            write_photons(str(tmp_path / ('photons_%d.npz' % r)), part)
        text = open(cfg).read().replace('in_photons_file = photons.npz',
                                        'in_photons_file = photons_{rank}.npz')
        cfg = str(tmp_path / 'config_sharded.ini')
        open(cfg, 'w').write(text)
    prefix = str(tmp_path / 'sharded')
    _run_ranks(tmp_path, cfg, model_path, prefix)
    for it, (rmax, m) in enumerate(want, 1):
        assert np.array_equal(np.load(prefix + '_rmax%d.npy' % it), rmax)
        assert np.array_equal(np.load(prefix + '_model%d.npy' % it), m)
    assert np.array_equal(want[0][0], g['rmax_1'])
