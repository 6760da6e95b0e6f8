"""Posterior normalisation and merge on the GPU (rows a9, a10) vs the FP64
oracle and vs the reference's own merge_all / slice_merge kernels
(kernels.cu:84-152, which emc.py loads but never launches) run on the
golden posteriors (merge_num / merge_den of tests/golden/case_*.npz)."""
import numpy as np
import pytest
import torch

from helpers import GOLDEN_CASES, golden_dataset, golden_states, load_golden
from oracle import emc_oracle as E

pytestmark = pytest.mark.gpu

RTOL = 1e-10   # FP64 accumulators; atomics reorder the sums


def _setup(g, form):
    from rspi.device import DevicePhotons, EStep, Merge
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']))
    _, pm = E.generate_masks(size)
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form=form)
    return ds, es, Merge(es)


@pytest.mark.parametrize('form', ['fp64', 'screen'])
@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_merge_matches_oracle(name, form):
    g = load_golden(name)
    ds, es, mg = _setup(g, form)
    size, num_rot = int(g['size']), int(g['num_rot'])
    es.run(torch.from_numpy(g['model_in_1']).cuda())
    es.reduce()
    intens = mg.run().cpu().numpy()
    prob = g['prob_1']
    logz, post = E.posterior(prob)
    want, num, den = E.merge(post, ds, E.get_scales(ds, bool(g['need_scaling'])),
                             es.n_states0, num_rot, size)
    np.testing.assert_allclose(mg.num.cpu().numpy(), num, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(mg.den.cpu().numpy(), den, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(intens, want, rtol=1e-9, atol=1e-12)
    assert np.all(intens[den == 0] == 0)
    # the reference kernels' merge of the same posteriors
    np.testing.assert_allclose(mg.num.cpu().numpy(), g['merge_num'], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(mg.den.cpu().numpy(), g['merge_den'], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_posterior_normalisation(name):
    g = load_golden(name)
    _, es, mg = _setup(g, 'fp64')
    es.run(torch.from_numpy(g['model_in_2']).cuda())
    _, _, logz = es.reduce()
    post = torch.exp(es.frame_prob() - logz[None, :]).cpu().numpy()
    want_logz, want = E.posterior(g['prob_2'])
    np.testing.assert_allclose(logz.cpu().numpy(), want_logz, rtol=1e-12)
    np.testing.assert_allclose(post, want, rtol=1e-9, atol=1e-300)
    np.testing.assert_allclose(post.sum(0), 1., rtol=1e-12)


def test_coverage_is_rotation_adjoint_of_ones():
    from rspi import geometry
    from rspi.device import call, cur_stream, ptr
    size, num_rot = 21, 4
    rot = torch.from_numpy(geometry.emc_rotation_table(num_rot)).cuda()
    cov = torch.empty((num_rot, size * size), dtype=torch.float64, device='cuda')
    call('rspi_merge_coverage', num_rot, ptr(rot), size, ptr(cov), cur_stream())
    for j in range(num_rot):
        model = np.zeros(size * size)
        wts = np.zeros(size * size)
        E.slice_merge(np.ones(size * size), j * np.pi / num_rot, size, model, wts)
        np.testing.assert_allclose(cov[j].cpu().numpy(), model, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize('graph', [False, True])
def test_emc_merge_option_writes_intens(tmp_path, graph):
    """[emc] merge = true: each iteration's posterior-weighted intensities
    (from the E-step on the iteration's start model, the rescoring window
    defaulting to 20 nats) equal the oracle's merge of the golden posteriors
    and are written to output_%03d.h5 as intens; graph replays give the
    eager values."""
    import os
    from emc import EMC
    from helpers import write_case
    from rspi import h5lite
    g = load_golden('case_b')
    cfg = write_case(str(tmp_path), g, extra='merge = true\ncuda_graph = %s\n' % graph)
    rec = EMC(cfg)
    assert rec.screen_delta == 20.
    rec.model = g['model_in_1'].copy()
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    for it in (1, 2):
        rec.run_iteration(it)
        _, post = E.posterior(g['prob_%d' % it])
        want, _, _ = E.merge(post, ds, E.get_scales(ds, bool(g['need_scaling'])),
                             rec.estep.n_states0, num_rot, size)
        got = rec.intens.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
        out = h5lite.read_datasets(os.path.join(str(tmp_path), 'out', 'output_%03d.h5' % it))
        assert np.array_equal(out['intens'], got)
