"""The polar grid search of the per-pixel NLL (the comparison for L-BFGS) and
the model-update comparison (pattern search, grid, L-BFGS) on NLL and FRC."""
import numpy as np
import pytest
import torch

from helpers import random_photons
from oracle import adjoint_oracle as A
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M

pytestmark = pytest.mark.gpu


def test_grid_search_matches_oracle():
    """Per pixel: the chosen point's NLL equals the frame-by-frame oracle's
    minimum over the same 64 x 32 polar grid (1e-9 relative), and the chosen
    index is the oracle's wherever the two best values are not tied."""
    from rspi import geometry
    from rspi.device import DevicePhotons, MStep
    size, n, num_rot = 23, 40, 6
    d = random_photons(size, n, 30. * size, 31)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, True)
    ph = DevicePhotons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                       d['count_multi'], size * size, True)
    rng = np.random.default_rng(4)
    states = np.array([[sx, sy, dia] for sx in (-1., 0., 1.) for sy in (0., 1.) for dia in (2., 3.)])
    rmax = rng.integers(0, len(states) * num_rot, n).astype('i4')
    ms = MStep(ph, size)
    ms.frame_params_from_rmax(torch.from_numpy(rmax).cuda(), num_rot, len(states))
    rot = torch.from_numpy(geometry.phaser_rotation_table(np.arange(num_rot) * np.pi / num_rot)).cuda()
    sv = torch.from_numpy(states).cuda()
    scale = torch.from_numpy(rng.uniform(0.5, 2., n)).cuda()
    model = rng.random(size * size) + 1j * rng.random(size * size)
    f = torch.from_numpy(model.copy()).cuda()
    best = ms.grid(f, sv, rot, scale).cpu().numpy()
    got = f.cpu().numpy()
    kmat = E.sparse_frames(ds)
    qx, qy, qrad, mask, _ = M.get_qvals(size)
    ang = (rmax % num_rot) * np.pi / num_rot
    st = states[rmax // num_rot]
    s_np = scale.cpu().numpy()
    main = ms.main.cpu().numpy()
    agree = 0
    for i, t in enumerate(main):
        k = M.photons_pixel(kmat, ang, int(t), size, qx, qy)
        fr = M.fref_pixel(int(t), qx, qy, qrad, st[:, 2], st[:, :2])
        fo, nll_o, _ = A.grid_pixel(k, fr, s_np)
        assert abs(best[i] - nll_o) <= 1e-9 * max(1., abs(nll_o)), (t, best[i], nll_o)
        agree += np.isclose(got[t], fo, rtol=1e-12, atol=1e-14)
    assert agree >= 0.99 * main.size
    untouched = np.ones(size * size, bool)
    untouched[main] = False
    assert np.array_equal(got[untouched], model[untouched])


def test_compare_updates_nll_and_frc():
    """From a perturbed start: L-BFGS lowers the NLL, refining the grid
    result lowers it further, and the refined model correlates better with
    the truth than the start (FRC)."""
    from rspi import synth
    from rspi.device import DevicePhotons, EStep
    from rspi.evaluate import compare_updates
    size, n, num_rot = 41, 400, 36
    data = synth.generate(size, n, 600., 8, 6., 0.3, (6., 8.), 2., seed=12)
    ph = DevicePhotons(data['ones'], data['multi'], data['place_ones'], data['place_multi'],
                       data['count_multi'], size * size, True)
    truth = data['fsample'] / float(data['rel_scale'])
    sx, sy, dia, nst = E.generate_states(E.parse_triple('-2 2 5'), E.parse_triple('-2 2 5'),
                                         E.parse_triple('6 8 3'))
    _, pm = E.generate_masks(size)
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, np.zeros(size * size), form='fp64')
    es.run(torch.from_numpy(truth).cuda())
    _, rmax, _ = es.reduce()
    from rspi import geometry
    sv = torch.from_numpy(geometry.state_values(sx, sy, dia, nst)).cuda()
    rng = np.random.default_rng(3)
    start = truth * (1 + 0.3 * rng.standard_normal(truth.size)) + \
        0.3 * np.abs(truth).mean() * (rng.standard_normal(truth.size) + 1j * rng.standard_normal(truth.size))
    out = compare_updates(ph, size, start, truth, rmax, num_rot, sv, lbfgs_steps=40)
    nll = out['nll']
    assert nll['lbfgs'] < nll['start']
    assert nll['grid_lbfgs'] <= nll['grid'] + 1e-9 * abs(nll['grid'])
    for k, f in out['frc'].items():
        assert np.all(np.isfinite(f)) and np.all(np.abs(f) <= 1 + 1e-12), k
    assert out['frc_mean']['grid_lbfgs'] > out['frc_mean']['start']
    print({k: round(v, 4) for k, v in out['frc_mean'].items()}, nll)
