"""The reference phaser's per-pixel, per-frame methods (get_photons_pixel,
get_fref_d, get_pixel_constants, get_rescale_pixel, get_logq_pixel,
iterate_pixel_pattern, run_pixel_pattern, _get_sphere, get_fcalc_all and
the photons CSR matrix) on the device against the FP64 oracle."""
import os

import numpy as np
import pytest
import torch

from helpers import load_golden, random_photons, write_case
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M

pytestmark = pytest.mark.gpu


def _phaser_case(tmp_path, size, n, seed, even=False):
    from maxLP import MaxLPhaser
    from rspi.photonfile import write_photons
    d = random_photons(size, n, 25. * size, seed, empty_frames=(1,))
    path = os.path.join(str(tmp_path), 'p.npz')
    write_photons(path, d)
    rng = np.random.default_rng(seed)
    sx = rng.choice([-1., 0., 1.], n)
    sy = rng.choice([0., 1.], n)
    dia = rng.choice([5., 7.], n)
    ang = rng.uniform(0., 2. * np.pi, n)
    model = (rng.random(size * size) + 1j * rng.random(size * size)) * 2.
    ph = MaxLPhaser(path, size=size)
    ph._run_phaser(model, sx, sy, dia, ang)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size)
    return ph, E.sparse_frames(ds), model, (sx, sy, dia, ang)


@pytest.mark.parametrize('size', [23, 16])
def test_pixel_frames_match_oracle(size, tmp_path):
    """k_d bit-exact (even sizes: the flat column x*size + size aliases the
    next row's first pixel, as in the reference's CSR lookup), fref_d to
    rounding, with all frames and with a subset."""
    ph, kmat, _, (sx, sy, dia, ang) = _phaser_case(tmp_path, size, 40, 3 + size)
    qx, qy, qrad, _, _ = M.get_qvals(size)
    shifts = np.stack([sx, sy], axis=1)
    pix = list(np.flatnonzero(ph.mask)[::7]) + [0, size * size - 1]
    for t in pix:
        k = ph.get_photons_pixel(None, t).cpu().numpy()
        assert np.array_equal(k, M.photons_pixel(kmat, ang, int(t), size, qx, qy)), t
        fr = ph.get_fref_d(None, t).cpu().numpy()
        np.testing.assert_allclose(fr, M.fref_pixel(int(t), qx, qy, qrad, dia, shifts),
                                   rtol=1e-13, atol=1e-15)
    sub = np.array([5, 0, 17, 39, 5])
    t = int(np.flatnonzero(ph.mask)[3])
    k = ph.get_photons_pixel(sub, t).cpu().numpy()
    assert np.array_equal(k, M.photons_pixel(kmat, ang, t, size, qx, qy)[sub])


def test_pixel_values_and_pattern_match_oracle(tmp_path):
    size = 21
    ph, kmat, model, (sx, sy, dia, ang) = _phaser_case(tmp_path, size, 60, 8)
    qx, qy, qrad, _, _ = M.get_qvals(size)
    shifts = np.stack([sx, sy], axis=1)
    pattern = M.gen_pattern(8)
    for t in np.flatnonzero(ph.mask)[::11][:6]:
        t = int(t)
        k = M.photons_pixel(kmat, ang, t, size, qx, qy)
        fr = M.fref_pixel(t, qx, qy, qrad, dia, shifts)
        const = ph.get_pixel_constants(t)
        f0 = complex(model[t])
        cand = f0 + pattern * abs(f0) / 4.
        np.testing.assert_allclose(ph.get_rescale_pixel(cand, t, const).cpu().numpy(),
                                   M.rescale_pixel(cand, k, fr), rtol=1e-12)
        np.testing.assert_allclose(ph.get_logq_pixel(cand, t, const=const).cpu().numpy(),
                                   M.logq_pixel(cand, k, fr), rtol=1e-11, atol=1e-12)
        np.testing.assert_allclose(ph.get_logq_pixel(cand, t, rescale=0.7, const=const)
                                   .cpu().numpy(), M.logq_pixel(cand, k, fr, 0.7),
                                   rtol=1e-11, atol=1e-12)
        got = ph.run_pixel_pattern(model, t)
        want = M.run_pixel_pattern(f0, k, fr, pattern, None, 10)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
        got = ph.run_pixel_pattern(torch.from_numpy(model), t, rescale=0.9)
        want = M.run_pixel_pattern(f0, k, fr, pattern, 0.9, 10)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)


def test_photons_csr_and_sphere(tmp_path):
    size = 19
    ph, kmat, model, _ = _phaser_case(tmp_path, size, 30, 2)
    assert np.array_equal(ph.photons.to_dense().cpu().numpy(), np.asarray(kmat.todense()))
    qx, qy, qrad, _, _ = M.get_qvals(size)
    sval = np.pi * qrad * 6.5
    sphere = (np.sin(sval) - sval * np.cos(sval)) / sval ** 3
    np.testing.assert_allclose(ph._get_sphere(6.5).cpu().numpy().ravel(), sphere, rtol=1e-13)
    want = model + sphere * np.exp(1j * 2 * np.pi * (qx * 1.5 + qy * -0.5))
    got = ph.get_fcalc_all(model, 6.5, (1.5, -0.5)).cpu().numpy().ravel()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)


def test_pixel_api_needs_frame_parameters(tmp_path):
    from maxLP import MaxLPhaser
    g = load_golden('case_a')
    write_case(str(tmp_path), g)
    ph = MaxLPhaser(os.path.join(str(tmp_path), 'photons.npz'), size=int(g['size']))
    with pytest.raises(ValueError):
        ph.get_pixel_constants(int(np.flatnonzero(ph.mask)[0]))


def test_emc_sphere_and_ramp(tmp_path):
    """EMC.sphere / EMC.ramp (emc.py:244-254) on the device against the
    reference's NumPy expressions on the same integer-centred grids."""
    from emc import EMC
    g = load_golden('case_a')
    rec = EMC(write_case(str(tmp_path), g))
    size = rec.size
    x, y = np.indices((size, size), dtype='f8')
    x = x.ravel() - size // 2
    y = y.ravel() - size // 2
    rad = np.sqrt(x * x + y * y)
    for n in (0, len(rec.sphere_dia) - 1):
        want = np.exp(1j * 2. * np.pi * (x * rec.shiftx[n] + y * rec.shifty[n]) / size)
        np.testing.assert_allclose(rec.ramp(n).cpu().numpy(), want, rtol=1e-13, atol=1e-15)
        _check_sphere(rec.sphere(n).cpu().numpy(), rad, rec.sphere_dia[n], size)
    _check_sphere(rec.sphere(None, 7.25).cpu().numpy(), rad, 7.25, size)


def _check_sphere(got, rad, dia, size):
    s = np.pi * rad * dia / size
    s[s == 0] = 1.e-5
    want = (np.sin(s) - s * np.cos(s)) / s ** 3
    # sin s - s cos s cancels to s^3/3 at the centre (s = 1e-5): one ulp of
    # sin there is ~5e-6 of the difference, in either library
    far = s > 1.e-3
    np.testing.assert_allclose(got[far], want[far], rtol=1e-12)
    np.testing.assert_allclose(got[~far], want[~far], rtol=1e-4)


def test_pixel_api_follows_the_last_run(tmp_path):
    """A second _run_phaser with other frame parameters: the per-pixel API
    uses the new ones."""
    size = 17
    ph, kmat, model, (sx, sy, dia, ang) = _phaser_case(tmp_path, size, 30, 4)
    qx, qy, qrad, _, _ = M.get_qvals(size)
    ang2 = (ang + 0.7) % (2 * np.pi)
    dia2 = dia + 0.5
    ph._run_phaser(model, sx, sy, dia2, ang2)
    t = int(np.flatnonzero(ph.mask)[5])
    assert np.array_equal(ph.get_photons_pixel(None, t).cpu().numpy(),
                          M.photons_pixel(kmat, ang2, t, size, qx, qy))
    np.testing.assert_allclose(ph.get_fref_d(None, t).cpu().numpy(),
                               M.fref_pixel(t, qx, qy, qrad, dia2, np.stack([sx, sy], 1)),
                               rtol=1e-13, atol=1e-15)
