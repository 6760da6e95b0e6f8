"""bench.py's input files on CPU: the configuration file it writes for the
reconstruction (single job and frame-sharded ranks) parses and names the
workload's geometry, state grid and options."""
import configparser
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize('rank', [None, 1])
def test_write_inputs_config(tmp_path, rank):
    sys.path.insert(0, REPO)
    import bench
    w = bench.workload(1, 8)
    data = bench.generate_data(1, w)
    cfg = bench.write_inputs(str(tmp_path), w, data, 'screen', 2.5, 20., 'sets', 'pattern',
                             False, rank=rank, slice_math='fp32', set_order='rank')
    c = configparser.ConfigParser()
    c.read(cfg)
    e = c['emc']
    assert int(e['size']) == w['size']
    assert int(e['num_rot']) == w['num_rot']
    assert int(e['num_modes']) == w['n_modes']
    assert e['sphere_dia'] == w['recon']['sphere_dia']
    assert e['shiftx'] == w['recon']['shiftx'] and e['shifty'] == w['recon']['shifty']
    assert e['form'] == 'screen' and float(e['slice_budget_gb']) == 2.5
    assert float(e['screen_delta']) == 20.
    assert e['kernel'] == 'sets' and e['mstep'] == 'pattern' and e['slice_math'] == 'fp32'
    assert e['set_order'] == 'rank'
    assert e['autotune'] == 'False'
    if rank is None:
        assert e['in_photons_file'] == 'photons.npz'
        assert os.path.exists(os.path.join(str(tmp_path), 'photons.npz'))
    else:
        # each rank reads its own file; the reconstruction substitutes {rank}
        assert e['in_photons_file'] == 'photons_{rank}.npz'
        assert os.path.exists(os.path.join(str(tmp_path), 'photons_%d.npz' % rank))
    got = np.load(os.path.join(str(tmp_path), 'photons.npz' if rank is None
                               else 'photons_%d.npz' % rank))
    assert int(got['ones'].shape[0]) == 8
