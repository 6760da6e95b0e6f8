"""The FP32-screened MaxLP pattern search (rspi_maxlp_pattern_screened)
against the plain FP64 search (rspi_maxlp_pattern): bit-identical models and
ring rescales, the screen settling iterations; and the log2 error bound the
screen relies on, checked over every float of its range."""
import os

import numpy as np
import pytest
import torch

from helpers import load_golden, random_photons, write_case

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint64 if a.dtype.itemsize == 8 else np.uint8)


def test_log2_bound_holds_for_every_float():
    """lg2.approx.f32 against FP64 log2 over every float in [2^-100, 2^100]:
    within 2^-21 + 2^-22 |lg2(x)|, the bound used for each FP32 term."""
    from rspi.device import cur_stream, ptr
    from rspi.lib import check, load
    out = torch.zeros(2, dtype=torch.float64, device='cuda')
    check(load().rspi_log2_error_max(2.0 ** -100, 2.0 ** 100, ptr(out), cur_stream()), 'log2')
    torch.cuda.synchronize()
    ratio, eabs = out.cpu().numpy()
    print('log2 error: %.3f of the bound, largest absolute %.3g' % (ratio, eabs))
    assert 0. < ratio <= 1.


def _run_both(path, size, params, model, modes=None, num_modes=1):
    from maxLP import MaxLPhaser
    res = {}
    for screen in (False, True):
        ph = MaxLPhaser(path, size=size, screen=screen, num_modes=num_modes)
        out = ph._run_phaser(model, *params, modes=modes)
        torch.cuda.synchronize()
        res[screen] = (out, ph.mstep.rescales.cpu().numpy(), ph.mstep.stats.cpu().numpy())
    return res


def _check_same(res):
    assert np.array_equal(_bits(res[False][0]), _bits(res[True][0]))
    assert np.array_equal(_bits(res[False][1]), _bits(res[True][1]))
    st = res[True][2]
    print('screened iterations %d, FP64 iterations %d, finalists %d' % tuple(st))
    return st


def _random_case(tmp_path, size, n, n_states, seed, mean_factor=30.):
    from rspi.photonfile import write_photons
    d = random_photons(size, n, mean_factor * size, seed, empty_frames=(1,))
    path = os.path.join(str(tmp_path), 'p.npz')
    write_photons(path, d)
    rng = np.random.default_rng(seed)
    states = np.stack([rng.uniform(-2., 2., n_states), rng.uniform(-2., 2., n_states),
                       rng.uniform(4., 8., n_states)], axis=1)
    pick = rng.integers(0, n_states, n)
    ang = rng.integers(0, 12, n) * np.pi / 12
    params = (states[pick, 0], states[pick, 1], states[pick, 2], ang)
    return path, params, rng


@pytest.mark.parametrize('size,n,n_states', [(23, 300, 12), (41, 800, 60), (61, 3000, 400)])
def test_screened_search_bit_identical(size, n, n_states, tmp_path):
    path, params, rng = _random_case(tmp_path, size, n, n_states, 7 + size)
    model = (rng.random(size * size) + 1j * rng.random(size * size)) * 3.
    st = _check_same(_run_both(path, size, params, model))
    assert st[0] > 0


def test_screened_search_modes_bit_identical(tmp_path):
    size, n, nm = 31, 900, 3
    path, params, rng = _random_case(tmp_path, size, n, 30, 5)
    model = (rng.random((nm, size * size)) + 1j * rng.random((nm, size * size))) * 2.
    modes = rng.integers(0, nm, n).astype('i4')
    st = _check_same(_run_both(path, size, params, model, modes=modes, num_modes=nm))
    assert st[0] > 0


def test_screen_falls_back_beyond_one_chunk(tmp_path):
    """More than 1024 (shift, diameter) states: no shared-memory copy of the
    populated states, every iteration runs the FP64 pass."""
    size, n = 19, 1100
    path, params, rng = _random_case(tmp_path, size, n, 100000, 3)
    model = rng.random(size * size) + 1j * rng.random(size * size)
    res = _run_both(path, size, params, model)
    st = _check_same(res)
    assert st[0] == 0 and st[1] > 0
    # the chunked path against the oracle's phaser: the ring pass in full
    # (its mean rescale enters every main pixel), a sample of main pixels.
    # The main pass covers the ring pixels too, so only the sampled main
    # pixels hold the same values in both.
    from oracle import emc_oracle as E
    from oracle import maxlp_oracle as M
    d = random_photons(size, n, 30. * size, 3, empty_frames=(1,))
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size)
    _, _, _, mask, rmask = M.get_qvals(size)
    main = np.flatnonzero(mask)[::9]
    assert np.any(rmask[main])
    want = M.run_phaser(model, E.sparse_frames(ds), *params, size, pixels=main)
    got = np.asarray(res[False][0]).ravel()
    np.testing.assert_allclose(got[main], want[main], rtol=1e-9, atol=1e-12)


def test_screen_handles_zero_model(tmp_path):
    """A zero start model (the pattern's step is 0): the searches agree."""
    size, n = 17, 200
    path, params, _ = _random_case(tmp_path, size, n, 8, 11)
    model = np.zeros(size * size, complex)
    _check_same(_run_both(path, size, params, model))


def test_emc_golden_screen_on_off_bit_identical(tmp_path):
    from emc import EMC
    g = load_golden('case_a')
    models = {}
    for screen in (False, True):
        d = os.path.join(str(tmp_path), str(screen))
        cfg = write_case(d, g, extra='form = screen\nphaser_screen = %s\n' % screen)
        rec = EMC(cfg)
        rec.model = g['model_in_1'].copy()
        for it in range(3):
            rec.run_iteration(None)
        models[screen] = (rec.model.copy(), rec.rmax.copy())
    assert np.array_equal(_bits(models[False][0]), _bits(models[True][0]))
    assert np.array_equal(models[False][1], models[True][1])


def test_emc_synthetic_screen_on_off_bit_identical(tmp_path):
    """Seeded synthetic frames with the 101^2 / 245-state geometry (400
    frames): two EMC iterations with and without the screen give the same
    model bits and argmax."""
    from emc import EMC
    from rspi import synth
    from rspi.photonfile import write_photons
    c = synth.CONFIGS[1]
    r = c['recon']
    n = 400
    data = synth.generate(c['size'], n, c['mean_count'], c['n_blobs'], c['obj_radius'],
                          c['fluence_sigma'], c['dia'], c['shift_max'], seed=20260001,
                          **synth.config_extras(1))
    model0 = synth.initial_model(c['size'], 20260102)
    out = {}
    for screen in (False, True):
        d = os.path.join(str(tmp_path), str(screen))
        os.makedirs(os.path.join(d, 'out'))
        write_photons(os.path.join(d, 'photons.npz'), data)
        cfg = os.path.join(d, 'config.ini')
        with open(cfg, 'w') as f:
            f.write('[emc]\nsize = %d\nin_photons_file = photons.npz\noutput_folder = out/\n'
                    'log_file = out/EMC.log\nneed_scaling = True\nnum_rot = %d\n'
                    'sphere_dia = %s\nshiftx = %s\nshifty = %s\nform = screen\n'
                    'phaser_screen = %s\n' % (c['size'], r['num_rot'], r['sphere_dia'],
                                              r['shiftx'], r['shifty'], screen))
        rec = EMC(cfg)
        rec.model = model0.copy().reshape(rec._model_shape())
        for it in range(2):
            rec.run_iteration(None)
        out[screen] = (rec.model.copy(), rec.rmax.copy(), rec.phaser.mstep.stats.cpu().numpy())
    assert np.array_equal(_bits(out[False][0]), _bits(out[True][0]))
    assert np.array_equal(out[False][1], out[True][1])
    st = out[True][2]
    print('screened iterations %d, FP64 iterations %d, finalists %d' % tuple(st))
    assert st[0] > st[1]
