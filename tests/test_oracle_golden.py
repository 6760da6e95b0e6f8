"""The FP64 oracle against golden vectors from the reference's own code.

The goldens come from tests/golden/make_golden.py, which runs the reference
emc.py / maxLP.py / dset.py unmodified (NumPy standing in for CuPy, the
reference kernels.cu compiled for the CPU).  These checks pin the oracle;
the GPU tests then compare the CUDA path with the pinned oracle.
"""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, golden_dataset, golden_states, load_golden
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M


@pytest.fixture(params=GOLDEN_CASES, scope='module')
def gold(request):
    return load_golden(request.param)


def test_dataset_bit_exact(gold):
    ds = golden_dataset(gold)
    assert ds['ones_accum'].dtype == np.int64
    assert np.array_equal(ds['ones_accum'], gold['ds_ones_accum'])
    assert np.array_equal(ds['multi_accum'], gold['ds_multi_accum'])
    assert ds['mean_count'] == float(gold['ds_mean_count'])
    if 'ds_counts' in gold:
        assert np.array_equal(ds['counts'], gold['ds_counts'])
    assert np.array_equal(E.get_powder(ds), gold['ds_powder'])
    assert np.array_equal(E.get_scales(ds, bool(gold['need_scaling'])), gold['scales'])


def test_holo_and_rotated_slices(gold):
    ds = golden_dataset(gold)
    size, num_rot = int(gold['size']), int(gold['num_rot'])
    sx, sy, dia, _ = golden_states(gold)
    for r in range(gold['holo'].shape[0]):
        w = E.holo_slice(gold['model0'], sx[r], sy[r], dia[r], 1., 1., size, ds['bg'])
        np.testing.assert_allclose(w, gold['holo'][r], rtol=1e-14, atol=0)
        for k, j in enumerate((0, 1, num_rot - 1)):
            lv = E.rotate_slice(gold['holo'][r], j * np.pi / num_rot, 1., size, ds['bg'], 1)
            np.testing.assert_allclose(lv, gold['rotlog'][3 * r + k], rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize('it', [1, 2])
def test_prob_argmax_unravel(gold, it):
    ds = golden_dataset(gold)
    size, num_rot = int(gold['size']), int(gold['num_rot'])
    sx, sy, dia, ns = golden_states(gold)
    _, pm = E.generate_masks(size)
    scales = E.get_scales(ds, bool(gold['need_scaling']))
    prob, _, _ = E.calc_prob(gold['model_in_%d' % it], ds, sx, sy, dia, size, num_rot, pm, scales)
    np.testing.assert_allclose(prob, gold['prob_%d' % it], rtol=1e-12, atol=0)
    _, rmax = E.get_rmax(prob)
    assert np.array_equal(rmax, gold['rmax_%d' % it])
    un = np.stack(E.unravel_rmax(rmax, sx, sy, dia, ns, num_rot))
    assert np.array_equal(un, gold['unravel_%d' % it])


@pytest.mark.parametrize('it', [1, 2])
def test_phaser(gold, it):
    ds = golden_dataset(gold)
    size = int(gold['size'])
    kmat = E.sparse_frames(ds)
    fout, resc = M.run_phaser(gold['model_in_%d' % it], kmat, *gold['unravel_%d' % it], size,
                              return_rescale=True)
    np.testing.assert_allclose(resc, float(gold['rescale_%d' % it]), rtol=1e-13)
    np.testing.assert_allclose(fout, gold['model_out_%d' % it], rtol=1e-12, atol=1e-14)


def test_phaser_pixel_pieces(gold):
    ds = golden_dataset(gold)
    size = int(gold['size'])
    kmat = E.sparse_frames(ds)
    qx, qy, qrad, _, _ = M.get_qvals(size)
    for i, t in enumerate(gold['ph_pixels']):
        k = M.photons_pixel(kmat, gold['ph_ang'], int(t), size, qx, qy)
        assert np.array_equal(k, gold['ph_k'][i])
        fr = M.fref_pixel(int(t), qx, qy, qrad, gold['ph_diams'], gold['ph_shifts'])
        np.testing.assert_allclose(fr, gold['ph_fref'][i], rtol=1e-13, atol=1e-16)
        rs = M.rescale_pixel(gold['ph_cand'][i], k, fr)
        np.testing.assert_allclose(rs, gold['ph_rescale'][i], rtol=1e-13)
        lq = M.logq_pixel(gold['ph_cand'][i], k, fr, None)
        np.testing.assert_allclose(lq, gold['ph_logq'][i], rtol=1e-12, atol=1e-13)


def test_pattern_constants():
    pat = M.gen_pattern(8)
    assert pat.size == 1089 and pat[pat.size // 2] == 0
    assert pat[0] == -8 - 8j and pat[-1] == 8 + 8j


def test_posterior_normalises():
    rng = np.random.default_rng(0)
    prob = rng.normal(-1000., 30., size=(50, 7))
    logz, post = E.posterior(prob)
    np.testing.assert_allclose(post.sum(0), 1., rtol=1e-12)
    np.testing.assert_allclose(logz, np.log(np.exp(prob - prob.max(0)).sum(0)) + prob.max(0),
                               rtol=1e-14)


@pytest.mark.parametrize('name', ['case_a', 'case_b', 'phase_a'])
def test_phase_oracle_matches_reference(name):
    """The model-refinement restatement (oracle/phase_oracle.py) against the
    reference's own MaxLPhaser._improve_model / diffmap / er / _get_support
    run on the same inputs (tests/golden/make_golden.py)."""
    import os
    from conftest import GOLDEN
    from oracle import phase_oracle as P
    g = np.load(os.path.join(GOLDEN, name + '.npz'))
    size = int(g['size'])
    f = g['phase_in']
    inv = P.get_invmask(size)
    assert np.array_equal(inv, g['phase_invmask'])
    supp = P.get_support(f, size)
    assert np.array_equal(supp, g['phase_supp'])
    np.testing.assert_array_equal(P.diffmap(f, f, inv, supp, size), g['phase_dm1'])
    np.testing.assert_array_equal(P.er(f, f, inv, supp, size), g['phase_er1'])
    out, _ = P.improve_model(f, size)
    np.testing.assert_array_equal(out, g['phase_out'])
    if name == 'phase_a':
        assert 0.5 < supp.mean() < 0.99   # a proper support, not the whole image


@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_emc_nll_oracle_matches_reference_likelihood(name):
    """The differentiable E-step NLL restatement at grid values equals minus
    the reference's likelihood of each frame in its argmax state, plus the
    Poisson term K_d log s_d (oracle/adjoint_oracle.emc_nll_torch)."""
    import torch
    from oracle import adjoint_oracle as A
    g = load_golden(name)
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    _, pm = E.generate_masks(size)
    scales = E.get_scales(ds, bool(g['need_scaling']))
    model = g['model_in_1']
    rmax = g['rmax_1']
    s0, j = rmax // num_rot, rmax % num_rot
    _, vscale = E.msum_vscale(model, sx, sy, dia, size, ds['bg'], pm, E.get_powder(ds))
    t = lambda a: torch.tensor(np.asarray(a, dtype='f8'))  # noqa: E731
    val = float(A.emc_nll_torch(t(model.real), t(model.imag), t(dia[s0]), t(sx[s0]), t(sy[s0]),
                                t(scales), vscale, E.sparse_frames(ds), j * np.pi / num_rot,
                                size, ds['bg'], pm < 1))
    k_tot = np.asarray(E.sparse_frames(ds, pm < 1).sum(1)).ravel()
    want = -np.sum(g['prob_1'][rmax, np.arange(rmax.size)] + k_tot * np.log(scales))
    np.testing.assert_allclose(val, want, rtol=1e-12)


@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_merge_oracle_matches_reference_kernels(name):
    """oracle/emc_oracle.merge (num, den) against the reference's own
    merge_all + slice_merge kernels (kernels.cu:84-152) on the same
    posteriors (tests/golden/make_golden.py), and the oracle's posterior
    against the goldens' normalisation."""
    g = load_golden(name)
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    n0 = g['prob_1'].shape[0] // num_rot
    _, post = E.posterior(g['prob_1'])
    np.testing.assert_allclose(np.where(post >= E.P_MIN, post, 0.), g['merge_post'],
                               rtol=1e-12, atol=1e-15)
    _, num, den = E.merge(g['merge_post'], ds, g['scales'], n0, num_rot, size)
    np.testing.assert_allclose(num, g['merge_num'], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(den, g['merge_den'], rtol=1e-13, atol=1e-15)
