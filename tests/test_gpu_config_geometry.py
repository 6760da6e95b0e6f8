"""Parity of the default screened form at the benchmark geometries.

The golden and random cases are small detectors.  These tests run the
screened E-step (its default kernel and the four-row quad kernel, with the
column-part split and frame ordering they choose on their own) on data
generated like the
benchmark's, at the 185x185 production geometry (24,912 likelihood pixels,
the full 9 x 9 x 5 state grid x 180 rotations) and at the 101x101 small
geometry (7 x 7 x 5 x 180), with more frames than one frame-ordering window:

* the screened FP32 likelihoods against the FP64 oracle (emc.py:159-205,
  kernels.cu:116-137) on a subset of (shift, diameter) states, every
  rotation and every frame: within 1e-5 relative;
* the FP64 form against the same oracle rows: within 1e-11;
* over the whole grid, the screened form's argmax equal to the FP64 form's
  (and to the oracle's on the subset), its maximum equal to 1e-15 and its
  log-sum-exp within the bound of its rescoring window.
"""
import numpy as np
import pytest
import torch

from oracle import emc_oracle as E

pytestmark = pytest.mark.gpu

RTOL_F32 = 1e-5
RTOL_F64 = 1e-11


def _setup(cfg, n_frames):
    from rspi import geometry, synth
    from rspi.device import DevicePhotons
    c = synth.CONFIGS[cfg]
    data = synth.generate_config(cfg, device='cuda', num_data=n_frames)
    data = {k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in data.items()}
    size = c['size']
    r = c['recon']
    sx, sy, dia, nst = geometry.state_grid(geometry.parse_triple(r['shiftx']),
                                          geometry.parse_triple(r['shifty']),
                                          geometry.parse_triple(r['sphere_dia']))
    ds = E.parse_photons(data['ones'], data['multi'], data['place_ones'], data['place_multi'],
                         data['count_multi'], size * size, True)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], size * size, True)
    model = synth.initial_model(size, 20260100 + cfg)
    return ds, ph, size, r['num_rot'], sx, sy, dia, model


@pytest.mark.parametrize('kernel', [None, 'quad4'])
@pytest.mark.parametrize('cfg,n_frames,parts', [(2, 700, 2), (1, 600, 1)])
def test_screened_form_at_config_geometry(cfg, n_frames, parts, kernel):
    from rspi.device import EStep
    ds, ph, size, num_rot, sx, sy, dia, model = _setup(cfg, n_frames)
    _, pm = E.generate_masks(size)
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='screen', kernel=kernel)
    ref = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='fp64')
    # the column split the kernel picks at this geometry
    assert es.wide['n_parts'] == parts
    dm = torch.from_numpy(model).cuda()
    es.run(dm)
    maxll, rmax, logz = es.reduce()
    ref.run(dm)
    maxll64, rmax64, logz64 = ref.reduce()
    torch.cuda.synchronize()
    ph.err.check('config geometry')

    # oracle rows: four (shift, diameter) states spread over the grid
    states = np.linspace(0, sx.size - 1, 4).astype(int)
    want, _, _ = E.calc_prob(model, ds, sx, sy, dia, size, num_rot, pm,
                             E.get_scales(ds, True), states=states)
    rows = np.concatenate([np.arange(s * num_rot, (s + 1) * num_rot) for s in states])
    got32 = es.frame_prob()[torch.from_numpy(rows).cuda()].double().cpu().numpy()
    got64 = ref.frame_prob()[torch.from_numpy(rows).cuda()].cpu().numpy()
    assert np.max(np.abs(got32 - want) / np.abs(want)) <= RTOL_F32
    assert np.max(np.abs(got64 - want) / np.abs(want)) <= RTOL_F64

    # whole grid: the screened argmax and maximum are the FP64 form's
    r32, r64 = rmax.cpu().numpy(), rmax64.cpu().numpy()
    assert np.array_equal(r32, r64)
    np.testing.assert_allclose(maxll.cpu().numpy(), maxll64.cpu().numpy(), rtol=1e-15)
    # argmax-only window: log Z takes the other states from their FP32
    # values, each within eps_d of FP64 (eps_d / |log Z| < 1e-6 here)
    np.testing.assert_allclose(logz.cpu().numpy(), logz64.cpu().numpy(), rtol=1e-6)
    # on the oracle's rows, frames whose best state lies there agree with it
    sub_best = want.max(0)
    full_best = maxll64.cpu().numpy()
    on_sub = sub_best >= full_best
    assert np.array_equal(rows[np.argmax(want, 0)][on_sub], r64[on_sub])
    # the whole FP32 matrix against the FP64 form's, every entry
    a = es.frame_prob().double()
    b = ref.frame_prob()
    rel = ((a - b).abs() / b.abs()).max().item()
    assert rel <= RTOL_F32, rel
