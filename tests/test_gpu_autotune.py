"""The likelihood kernel's autotuner: every candidate tiling gives the same
FP64-rescored argmax, maximum and log-sum-exp (bit for bit), the tuner picks
one of them and caches it per geometry, and EMC runs it by default."""
import json

import numpy as np
import pytest
import torch

from helpers import golden_dataset, golden_states, load_golden, write_case
from oracle import emc_oracle as E

pytestmark = pytest.mark.gpu


def _estep(g, **kw):
    from rspi.device import DevicePhotons, EStep
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']))
    _, pm = E.generate_masks(size)
    return EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], **kw)


@pytest.mark.parametrize('form,kernel', [('screen', 'sets'), ('screen', 'quad4'),
                                         ('screen', 'stream'), ('fp64', 'stream')])
def test_every_candidate_gives_the_same_rescored_results(form, kernel):
    from rspi import autotune
    g = load_golden('case_b')
    model = torch.from_numpy(g['model_in_2']).cuda()
    es = _estep(g, form=form, kernel=kernel)
    out = []
    for cfg in autotune.candidates(es):
        es.configure(**cfg)
        es.run(model)
        maxll, rmax, logz = es.reduce()
        torch.cuda.synchronize()
        out.append((cfg, rmax.cpu().numpy(), maxll.cpu().numpy(), logz.cpu().numpy()))
    assert len(out) >= 2
    for cfg, rmax, maxll, logz in out[1:]:
        assert np.array_equal(rmax, out[0][1]), cfg
        assert np.array_equal(maxll, out[0][2]), cfg
        if form == 'fp64':
            np.testing.assert_allclose(logz, out[0][3], rtol=1e-13)
    assert np.array_equal(out[0][1], g['rmax_2'])


def test_tuner_picks_a_candidate_and_caches_it(tmp_path, monkeypatch):
    from rspi import autotune
    monkeypatch.setattr(autotune, 'CACHE', str(tmp_path / 'tune.json'))
    g = load_golden('case_a')
    es = _estep(g, form='screen', kernel='sets')
    es.slices(torch.from_numpy(g['model_in_1']).cuda())
    cfg, ms, results = autotune.tune(es)
    assert cfg in autotune.candidates(es) and ms > 0 and len(results) >= 2
    assert es.warps == cfg['warps'] and es.parts() == cfg['screen_parts']
    table = json.load(open(str(tmp_path / 'tune.json')))
    assert table[autotune.key(es)]['config'] == cfg
    es2 = _estep(g, form='screen', kernel='sets')
    cfg2, _, res2 = autotune.tune(es2)
    assert cfg2 == cfg and res2 is None                  # from the cache
    assert es2.warps == cfg['warps'] and es2.parts() == cfg['screen_parts']


def test_emc_tunes_by_default(tmp_path, monkeypatch):
    from emc import EMC
    from rspi import autotune
    monkeypatch.setattr(autotune, 'CACHE', str(tmp_path / 'tune.json'))
    g = load_golden('case_a')
    rec = EMC(write_case(str(tmp_path), g=g))
    rec.model = g['model_in_1'].copy()
    rec.run_iteration(1)
    assert rec.tuning[0] in autotune.candidates(rec.estep)
    assert np.array_equal(rec.rmax, g['rmax_1'])
