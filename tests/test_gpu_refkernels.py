"""The reference's own kernels (kernels.cu, built for sm_100a by
oracle/ref_gpu/build.py) on the same GPU: they reproduce the golden
likelihoods and per-pixel MaxLP pieces, and the product's FP64 E-step and
MaxLP M-step equal them.  Skipped when the reference kernels were not built
(the reference tree was absent at build time)."""
import os

import numpy as np
import pytest
import torch

from helpers import GOLDEN_CASES, golden_dataset, golden_states, load_golden
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M

pytestmark = pytest.mark.gpu

REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle',
                       '_ref', 'libref_kernels_gpu.so')
needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB),
                               reason='reference kernels not built for the GPU')


def _ref_data(g, ds):
    from oracle.ref_gpu import replay
    size = int(g['size'])
    _, pm = E.generate_masks(size)
    return replay.RefData(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                          ds['count_multi'], size, ds['bg'],
                          E.get_scales(ds, bool(g['need_scaling'])), pm, torch.device('cuda'))


@needs_ref
@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_reference_kernels_on_gpu_reproduce_goldens(name):
    from oracle.ref_gpu import replay
    g = load_golden(name)
    ds = golden_dataset(g)
    sx, sy, dia, _ = golden_states(g)
    data = _ref_data(g, ds)
    lib = replay.load()
    for it in (1, 2):
        model = torch.from_numpy(g['model_in_%d' % it]).cuda()
        prob = replay.estep(lib, data, model, sx, sy, dia, int(g['num_rot']))
        torch.cuda.synchronize()
        np.testing.assert_allclose(prob.cpu().numpy(), g['prob_%d' % it], rtol=1e-12,
                                   atol=1e-12 * np.abs(g['prob_%d' % it]).max())
        assert np.array_equal(prob.argmax(0).cpu().numpy().astype('i4'), g['rmax_%d' % it])


@needs_ref
@pytest.mark.parametrize('form', ['fp64', 'screen'])
@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_product_estep_equals_reference_kernels(name, form):
    """The product's likelihoods against the reference's kernels on the same
    device: FP64 form to 1e-11, screened form's candidates in FP64, same
    argmax."""
    from oracle.ref_gpu import replay
    from rspi.device import DevicePhotons, EStep
    g = load_golden(name)
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    _, pm = E.generate_masks(size)
    data = _ref_data(g, ds)
    model = torch.from_numpy(g['model_in_1']).cuda()
    want = replay.estep(replay.load(), data, model, sx, sy, dia, num_rot).cpu().numpy()
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']))
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form=form)
    es.run(model)
    maxll, rmax, _ = es.reduce()
    torch.cuda.synchronize()
    if form == 'fp64':
        np.testing.assert_allclose(es.frame_prob().cpu().numpy(), want, rtol=1e-11,
                                   atol=1e-11 * np.abs(want).max())
    assert np.array_equal(rmax.cpu().numpy(), want.argmax(0).astype('i4'))
    np.testing.assert_allclose(maxll.cpu().numpy(), want.max(0), rtol=1e-11)


@needs_ref
@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_reference_pattern_search_on_gpu(name):
    """The reference's get_f_dt kernel + the CuPy steps of get_logq_pixel as
    torch operations reproduce the golden per-pixel pieces, and the whole
    per-pixel pattern search equals the oracle's."""
    from oracle.ref_gpu import replay
    g = load_golden(name)
    ds = golden_dataset(g)
    size = int(g['size'])
    data = _ref_data(g, ds)
    lib = replay.load()
    dev = torch.device('cuda')
    ang = torch.from_numpy(np.asarray(g['ph_ang'], dtype='f8')).to(dev)
    shifts = torch.from_numpy(np.asarray(g['ph_shifts'], dtype='f8')).to(dev)
    diams = torch.from_numpy(np.asarray(g['ph_diams'], dtype='f8')).to(dev)
    pat = replay.pattern(dev)
    qx, qy, _, _, _ = M.get_qvals(size)
    kmat = E.sparse_frames(ds)
    for i, t in enumerate(g['ph_pixels']):
        k_d, fr = replay.pixel_constants(data, int(t), ang, shifts, diams)
        assert np.array_equal(k_d.cpu().numpy(), g['ph_k'][i])
        np.testing.assert_allclose(fr.cpu().numpy(), g['ph_fref'][i], rtol=1e-13, atol=1e-16)
        cand = torch.from_numpy(np.asarray(g['ph_cand'][i])).to(dev)
        rs = replay.rescale_pixel(lib, cand, k_d, fr)
        np.testing.assert_allclose(rs.cpu().numpy(), g['ph_rescale'][i], rtol=1e-12)
        lq = replay.logq_pixel(lib, cand, k_d, fr, None)
        np.testing.assert_allclose(lq.cpu().numpy(), g['ph_logq'][i], rtol=1e-12, atol=1e-13)
        f0 = complex(g['model_in_1'][int(t)])
        got = replay.run_pixel_pattern(lib, f0, k_d, fr, pat, None, 10)
        k_np = M.photons_pixel(kmat, g['ph_ang'], int(t), size, qx, qy)
        want = M.run_pixel_pattern(f0, k_np, g['ph_fref'][i], M.gen_pattern(8), None, 10)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
