"""Model refinement (error reduction and difference map, maxLP.py:271-354)
on the GPU against the reference's own results (the goldens written by
running MaxLPhaser._improve_model of the reference, tests/golden/make_golden.py)
and the FP64 NumPy oracle.

Tolerances: the centred transforms are FP64 line DFTs (the host uses an
FFT), so single steps agree to ~1e-14 of the image's largest magnitude and
the 15-iteration refinement to 1e-10 of it; the support mask, a threshold
on a smoothed field whose closest value sits 1e-3 (relative) from the
threshold in these cases, must be identical."""
import numpy as np
import pytest
import torch

from conftest import GOLDEN
from helpers import load_golden
from oracle import phase_oracle as P

pytestmark = pytest.mark.gpu

CASES = ('case_a', 'case_b', 'phase_a')
TOL_STEP = 1e-12
TOL_REFINE = 1e-10


def _golden(name):
    import os
    g = np.load(os.path.join(GOLDEN, name + '.npz'))
    g = {k: g[k] for k in g.files}
    return g, int(g['size'])


def _dev(a, dtype=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(a)).to('cuda', dtype)


def _support(fconv, size):
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    supp = torch.empty(size * size, dtype=torch.uint8, device='cuda')
    work = torch.empty(8 * size * size, dtype=torch.float64, device='cuda')
    call('rspi_phase_support', ptr(fconv), size, 12., 0.5, 3., 12, 1.2e-4, ptr(supp), ptr(work),
         cur_stream())
    return supp


def _refine(fconv, invmask, supp, x, size, n_dm, n_er):
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    out = x.clone()
    work = torch.empty(8 * size * size, dtype=torch.float64, device='cuda')
    call('rspi_phase_refine', ptr(fconv), ptr(invmask), ptr(supp), ptr(out), ptr(work), size,
         n_dm, n_er, cur_stream())
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _close(got, want, tol):
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))


@pytest.mark.parametrize('size', [5, 21, 25, 61, 185, 200])
@pytest.mark.parametrize('inverse', [0, 1])
def test_centred_transform_matches_numpy(size, inverse):
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    rng = np.random.default_rng(size + 10 * inverse)
    x = rng.standard_normal(size * size) + 1j * rng.standard_normal(size * size)
    xin = _dev(x)
    out = torch.empty_like(xin)
    work = torch.empty_like(xin)
    call('rspi_cdft2', ptr(xin), ptr(out), ptr(work), size, inverse, cur_stream())
    want = (P.centered_ifft(x, size) if inverse else P.centered_fft(x, size)).ravel()
    _close(out.cpu().numpy(), want, 1e-13)


@pytest.mark.parametrize('name', CASES)
def test_support_matches_reference(name):
    g, size = _golden(name)
    supp = _support(_dev(g['phase_in']), size).cpu().numpy().astype(bool)
    assert np.array_equal(supp, g['phase_supp'])
    assert np.array_equal(supp, P.get_support(g['phase_in'], size))


@pytest.mark.parametrize('name', CASES)
def test_single_steps_match_reference(name):
    g, size = _golden(name)
    f = _dev(g['phase_in'])
    inv = _dev(g['phase_invmask'], torch.uint8)
    supp = _dev(g['phase_supp'], torch.uint8)
    _close(_refine(f, inv, supp, f, size, 1, 0), g['phase_dm1'], TOL_STEP)
    _close(_refine(f, inv, supp, f, size, 0, 1), g['phase_er1'], TOL_STEP)


@pytest.mark.parametrize('name', CASES)
def test_improve_model_matches_reference(name):
    g, size = _golden(name)
    f = _dev(g['phase_in'])
    inv = _dev(g['phase_invmask'], torch.uint8)
    supp = _support(f, size)
    _close(_refine(f, inv, supp, f, size, 10, 5), g['phase_out'], TOL_REFINE)
    want, _ = P.improve_model(g['phase_in'], size, g['phase_invmask'])
    np.testing.assert_array_equal(want, g['phase_out'])   # the oracle is pinned


def test_maxlp_phaser_improve_model_api(tmp_path):
    """MaxLPhaser._improve_model / proj_fourier / proj_real / er / diffmap /
    _get_support on the golden case's data give the reference's results."""
    from helpers import write_case
    g = load_golden('case_a')
    cfg = write_case(str(tmp_path), g=g)
    import configparser
    import os
    c = configparser.ConfigParser()
    c.read(cfg)
    from maxLP import MaxLPhaser
    ph = MaxLPhaser(os.path.join(str(tmp_path), c.get('emc', 'in_photons_file')),
                    size=int(g['size']))
    size = int(g['size'])
    assert np.array_equal(ph.minvmask.cpu().numpy(), g['phase_invmask'])
    f = g['phase_in']
    out = ph._improve_model(f).cpu().numpy()
    assert np.array_equal(ph.minvsuppmask.cpu().numpy().ravel(), g['phase_supp'])
    _close(out, g['phase_out'], TOL_REFINE)
    _close(ph.diffmap(f, f).cpu().numpy(), g['phase_dm1'], TOL_STEP)
    _close(ph.er(f, f).cpu().numpy(), g['phase_er1'], TOL_STEP)
    pf = ph.proj_fourier(f, np.zeros_like(f)).cpu().numpy()
    np.testing.assert_array_equal(pf, P.proj_fourier(f, np.zeros_like(f), g['phase_invmask']))
    pr = ph.proj_real(f).cpu().numpy()
    _close(pr, P.proj_real(f, g['phase_supp'], size), TOL_STEP)
