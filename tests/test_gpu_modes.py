"""Several models at once (``num_modes``, parsed at emc.py:59 and unused by
the reference): the (mode, state) pairs are the E-step's state list and
MaxLP searches each mode over the frames whose argmax chose it.  The oracle
for the E-step is ``calc_prob_modes``; for the M-step it is the single-model
``run_phaser`` restricted to each mode's frames."""
import os

import numpy as np
import pytest
import torch

from helpers import golden_dataset, golden_states, load_golden, write_case
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M

pytestmark = pytest.mark.gpu

RTOL_F64 = 1e-11    # FP64 pipeline vs FP64 oracle: summation order only
RTOL_MODEL = 1e-9   # FP64 pattern search: same path, rounding-level differences


def _models(g, n_modes, seed=0):
    """Mode 0 is the golden input model; the others are perturbed copies.
    With case_b and this seed the oracle's argmax splits the 30 frames 16/14
    between two modes, and no pattern-search step of either mode has two
    candidates closer than 1e-11 relative (a mode with very few frames has
    exact ties, where any rounding difference picks another candidate)."""
    rng = np.random.default_rng(seed)
    m0 = np.asarray(g['model_in_1'], dtype=np.complex128).ravel()
    out = [m0]
    for _ in range(1, n_modes):
        out.append(m0 * (1. + 0.05 * rng.standard_normal(m0.size)) +
                   0.05 * (rng.standard_normal(m0.size) + 1j * rng.standard_normal(m0.size)))
    return out


def _photons(ds, need_scaling):
    from rspi.device import DevicePhotons
    return DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                         ds['count_multi'], ds['num_pix'], need_scaling)


@pytest.mark.parametrize('form', ['fp64', 'screen'])
def test_estep_two_modes_matches_oracle(form):
    from rspi.device import EStep
    g = load_golden('case_b')
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    _, pm = E.generate_masks(size)
    models = _models(g, 2)
    ph = _photons(ds, bool(g['need_scaling']))
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form=form, n_modes=2)
    dm = torch.from_numpy(np.concatenate(models)).cuda()
    es.run(dm)
    maxll, rmax, logz = es.reduce()
    torch.cuda.synchronize()
    want, _, vs = E.calc_prob_modes(models, ds, sx, sy, dia, size, num_rot, pm,
                                    E.get_scales(ds, bool(g['need_scaling'])))
    assert es.n_rows == want.shape[0] == 2 * sx.size * num_rot
    np.testing.assert_allclose(float(es.vscale.item()), vs, rtol=RTOL_F64)
    if form == 'fp64':
        np.testing.assert_allclose(es.frame_prob().cpu().numpy(), want, rtol=RTOL_F64,
                                   atol=RTOL_F64 * np.abs(want).max())
    mx, am = E.get_rmax(want)
    assert np.array_equal(rmax.cpu().numpy(), am)            # argmax bit-exact
    np.testing.assert_allclose(maxll.cpu().numpy(), mx, rtol=RTOL_F64)
    lz, _ = E.posterior(want)
    np.testing.assert_allclose(logz.cpu().numpy(), lz, rtol=RTOL_F64)
    # both modes are chosen by some frame in this case
    modes = am // num_rot // sx.size
    assert set(np.unique(modes)) == {0, 1}


def _mode_phaser_case(g, n_modes, modes):
    """Per-frame state values of golden iteration 1, the given modes."""
    sxv, syv, diav, angv = g['unravel_1']
    return (np.asarray(sxv), np.asarray(syv), np.asarray(diav), np.asarray(angv),
            np.asarray(modes, dtype='i4'))


@pytest.mark.parametrize('n_modes,empty', [(2, False), (3, True)])
def test_run_phaser_modes_match_oracle(n_modes, empty, tmp_path):
    """Each mode's model after _run_phaser equals the oracle's single-model
    phaser over that mode's frames; a mode without frames is unchanged."""
    from maxLP import MaxLPhaser
    g = load_golden('case_b')
    size = int(g['size'])
    write_case(str(tmp_path), g)
    ph = MaxLPhaser(os.path.join(str(tmp_path), 'photons.npz'), size=size, num_modes=n_modes)
    n = ph.num_data
    rng = np.random.default_rng(11)
    used = n_modes - 1 if empty else n_modes
    modes = rng.integers(0, used, n)
    modes[:used] = np.arange(used)
    sxv, syv, diav, angv, modes = _mode_phaser_case(g, n_modes, modes)
    models = np.stack(_models(g, n_modes))
    out = ph._run_phaser(models, sxv, syv, diav, angv, modes=modes)
    assert out.shape == models.shape
    kmat = E.sparse_frames(golden_dataset(g))
    for m in range(n_modes):
        sel = np.flatnonzero(modes == m)
        if sel.size == 0:
            assert np.array_equal(out[m], models[m])
            continue
        want = M.run_phaser(models[m], kmat[sel], sxv[sel], syv[sel], diav[sel], angv[sel], size)
        np.testing.assert_allclose(out[m], want, rtol=RTOL_MODEL, atol=1e-12)


def test_run_phaser_requires_modes_for_several_models(tmp_path):
    from maxLP import MaxLPhaser
    g = load_golden('case_a')
    write_case(str(tmp_path), g)
    ph = MaxLPhaser(os.path.join(str(tmp_path), 'photons.npz'), size=int(g['size']), num_modes=2)
    with pytest.raises(ValueError):
        ph._run_phaser(np.stack(_models(g, 2)), *g['unravel_1'])
    with pytest.raises(ValueError):
        ph._run_phaser(np.stack(_models(g, 2)), *g['unravel_1'], modes=np.full(ph.num_data, 2))


@pytest.mark.parametrize('form', ['fp64', 'screen'])
def test_emc_iteration_two_modes(form, tmp_path):
    """EMC with num_modes = 2: argmax from the oracle's multi-mode likelihood,
    each mode's MaxLP from the oracle over that mode's frames, and the
    output file's model/modes layout."""
    from emc import EMC
    from rspi import h5lite
    g = load_golden('case_b')
    cfg = write_case(str(tmp_path), g, extra='form = %s\n' % form)
    with open(cfg) as f:
        text = f.read().replace('num_modes = 1', 'num_modes = 2')
    with open(cfg, 'w') as f:
        f.write(text)
    rec = EMC(cfg)
    assert rec.model.shape == (2, int(g['size']) ** 2)
    models = _models(g, 2)
    rec.model = np.stack(models)
    rec.run_iteration(1)
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, nst = golden_states(g)
    _, pm = E.generate_masks(size)
    prob, _, _ = E.calc_prob_modes(models, ds, sx, sy, dia, size, num_rot, pm,
                                   E.get_scales(ds, bool(g['need_scaling'])))
    _, rmax = E.get_rmax(prob)
    assert np.array_equal(rec.rmax, rmax)
    modes = rmax // num_rot // sx.size
    r0 = rmax % (sx.size * num_rot)
    sxv, syv, diav, angv = E.unravel_rmax(r0, sx, sy, dia, nst, num_rot)
    kmat = E.sparse_frames(ds)
    for m in range(2):
        sel = np.flatnonzero(modes == m)
        want = models[m] if sel.size == 0 else \
            M.run_phaser(models[m], kmat[sel], sxv[sel], syv[sel], diav[sel], angv[sel], size)
        np.testing.assert_allclose(rec.model[m], want, rtol=RTOL_MODEL, atol=1e-12)
    out = h5lite.read_datasets(os.path.join(str(tmp_path), 'out', 'output_001.h5'))
    assert out['model'].shape == (2, size, size)
    assert np.array_equal(out['modes'], modes)
    np.testing.assert_array_equal(out['angles'], angv)
