"""Hand-written adjoints (row a16): the MaxLP negative log-likelihood and
the E-step likelihood through model slicing.

Each is checked against (1) torch autograd through the FP64 dense restatement in
oracle/adjoint_oracle.py, (2) FP64 central finite differences (step 1e-6)
on 64 random model pixels and every per-frame reference parameter, and (3)
torch.autograd.gradcheck of the autograd.Function."""
import os

import numpy as np
import pytest
import torch

from helpers import random_photons
from oracle import adjoint_oracle as A
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M

pytestmark = pytest.mark.gpu


def _case(size=21, n=30, seed=3):
    d = random_photons(size, n, 40. * size, seed)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size)
    rng = np.random.default_rng(seed)
    par = dict(dia=rng.uniform(2., 4., n), sx=rng.uniform(-1., 1., n),
               sy=rng.uniform(-1., 1., n), scale=rng.uniform(0.5, 2., n),
               ang=rng.uniform(0., np.pi, n))
    model = rng.random(size * size) + 1j * rng.random(size * size)
    return size, d, ds, par, model


def _problem(size, d, par, precision):
    from rspi.adjoint import NLLProblem
    from rspi.device import DevicePhotons
    ph = DevicePhotons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                       d['count_multi'], size * size)
    return NLLProblem(ph, size, par['ang'], precision=precision)


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype='f8')).cuda()


def test_fp64_value_and_gradient_match_autograd():
    size, d, ds, par, model = _case()
    pr = _problem(size, d, par, 'fp64')
    fre, fim = pr.model_pixels(model)
    val, g = pr.evaluate(fre, fim, _t(par['dia']), _t(par['sx']), _t(par['sy']),
                         _t(par['scale']), grad=True)
    k = A.photon_matrix(E.sparse_frames(ds), par['ang'], size, pr.pixels)
    ref = A.nll_and_grad(model[pr.pixels], par['dia'], par['sx'], par['sy'], par['scale'], k,
                         size, pr.pixels)
    np.testing.assert_allclose(float(val), ref[0], rtol=1e-12)
    got = [x.cpu().numpy() for x in g]
    np.testing.assert_allclose(got[0] + 1j * got[1], ref[1], rtol=1e-9, atol=1e-9)
    for a, b in zip(got[2:], ref[2:]):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-8)


def test_fp64_finite_differences():
    """Central differences, step 1e-6, on 64 random pixels (Re and Im) and
    every frame's diameter, shift and scale."""
    size, d, ds, par, model = _case(size=23, n=24, seed=4)
    pr = _problem(size, d, par, 'fp64')
    fre, fim = pr.model_pixels(model)
    args = [fre, fim, _t(par['dia']), _t(par['sx']), _t(par['sy']), _t(par['scale'])]
    _, g = pr.evaluate(*args, grad=True)
    h = 1e-6
    rng = np.random.default_rng(0)
    checks = [(0, i) for i in rng.choice(pr.n_pix, 64, replace=False)] + \
             [(1, i) for i in rng.choice(pr.n_pix, 64, replace=False)] + \
             [(j, i) for j in (2, 3, 4, 5) for i in range(len(par['dia']))]
    for j, i in checks:
        plus = [a.clone() for a in args]
        minus = [a.clone() for a in args]
        plus[j][i] += h
        minus[j][i] -= h
        fd = (float(pr.evaluate(*plus)) - float(pr.evaluate(*minus))) / (2 * h)
        an = float(g[j][i])
        assert abs(fd - an) <= 1e-5 * max(1., abs(an)), (j, i, fd, an)


def test_autograd_function_gradcheck():
    from rspi.adjoint import MaxLPNLL
    size, d, ds, par, model = _case(size=17, n=8, seed=5)
    pr = _problem(size, d, par, 'fp64')
    fre, fim = pr.model_pixels(model)
    inputs = [x.clone().requires_grad_(True) for x in
              (fre, fim, _t(par['dia']), _t(par['sx']), _t(par['sy']), _t(par['scale']))]
    # FP64 atomics make repeated backward passes differ in the last bits
    assert torch.autograd.gradcheck(lambda *a: MaxLPNLL.apply(*a, pr), inputs, eps=1e-6,
                                    atol=1e-4, rtol=1e-5, nondet_tol=1e-9)


def test_fp32_terms_close_to_fp64():
    size, d, ds, par, model = _case(seed=6)
    p32, p64 = _problem(size, d, par, 'fp32'), _problem(size, d, par, 'fp64')
    fre, fim = p64.model_pixels(model)
    args = [fre, fim, _t(par['dia']), _t(par['sx']), _t(par['sy']), _t(par['scale'])]
    v32, g32 = p32.evaluate(*args, grad=True)
    v64, g64 = p64.evaluate(*args, grad=True)
    assert abs(float(v32) - float(v64)) <= 1e-5 * abs(float(v64))
    for a, b in zip(g32, g64):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-3 * np.abs(b).max()


def test_lbfgs_decreases_nll():
    from rspi.adjoint import lbfgs_update
    size, d, ds, par, model = _case(seed=7)
    pr = _problem(size, d, par, 'fp64')
    fre, fim = pr.model_pixels(model)
    start = float(pr.evaluate(fre, fim, _t(par['dia']), _t(par['sx']), _t(par['sy']),
                              _t(par['scale'])))
    out, final, _ = lbfgs_update(pr, model, par['dia'], par['sx'], par['sy'], par['scale'],
                                 steps=30)
    assert final < start
    mask = np.zeros(size * size, bool)
    mask[pr.pixels] = True
    assert np.array_equal(out[~mask], model[~mask])


# ---------------------------------------------------------------------------
# E-step side: the likelihood through model slicing
# ---------------------------------------------------------------------------
def _emc_case(size=23, n=24, seed=7, num_rot=7):
    """Random frames with continuous per-frame parameters and orientations
    from the EMC rotation grid, a random model and a small background."""
    from rspi import geometry
    d = random_photons(size, n, 40. * size, seed)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size)
    rng = np.random.default_rng(seed)
    j = rng.integers(0, num_rot, n)
    par = dict(dia=rng.uniform(2., 4., n), sx=rng.uniform(-1., 1., n),
               sy=rng.uniform(-1., 1., n), scale=rng.uniform(0.5, 2., n),
               ang=j * np.pi / num_rot,
               rot_cs=geometry.emc_rotation_table(num_rot).reshape(-1, 2)[j])
    model = rng.random(size * size) + 1j * rng.random(size * size)
    bg = 0.01 * rng.random(size * size)
    _, pm = E.generate_masks(size)
    return size, d, ds, par, model, bg, pm, 0.37


def _emc_problem(size, d, par, pm, bg, vscale, precision):
    from rspi.adjoint import EMCNLLProblem
    from rspi.device import DevicePhotons
    ph = DevicePhotons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                       d['count_multi'], size * size)
    return EMCNLLProblem(ph, size, par['rot_cs'], pm, bg, vscale, precision=precision)


def _emc_args(model, par):
    m = torch.from_numpy(np.asarray(model)).cuda()
    return (m.real.contiguous(), m.imag.contiguous(), _t(par['dia']), _t(par['sx']),
            _t(par['sy']), _t(par['scale']))


def test_emc_nll_value_and_gradient_match_autograd():
    """FP64 E-step NLL and its adjoint against torch autograd through the
    dense FP64 restatement (oracle/adjoint_oracle.emc_nll_torch)."""
    size, d, ds, par, model, bg, pm, vscale = _emc_case()
    pr = _emc_problem(size, d, par, pm, bg, vscale, 'fp64')
    val, g = pr.evaluate(*_emc_args(model, par), grad=True)
    ref = A.emc_nll_and_grad(model, par['dia'], par['sx'], par['sy'], par['scale'], vscale,
                             E.sparse_frames(ds), par['ang'], size, bg, pm < 1)
    np.testing.assert_allclose(float(val), ref[0], rtol=1e-12)
    got = [x.cpu().numpy() for x in g]
    gm = got[0] + 1j * got[1]
    scale = np.abs(ref[1]).max()
    assert np.max(np.abs(gm - ref[1])) <= 1e-10 * scale
    for a, b in zip(got[2:], ref[2:]):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * np.abs(b).max())


def test_emc_nll_finite_differences():
    """FP64 central differences (step 1e-6) of the E-step NLL on 64 random
    model pixels (real and imaginary parts) and every per-frame diameter,
    shift and scale, against the adjoint."""
    size, d, ds, par, model, bg, pm, vscale = _emc_case(seed=8)
    pr = _emc_problem(size, d, par, pm, bg, vscale, 'fp64')
    args = list(_emc_args(model, par))
    _, g = pr.evaluate(*args, grad=True)
    g = [x.cpu().numpy() for x in g]
    h = 1e-6
    rng = np.random.default_rng(9)
    cand = np.flatnonzero(np.abs(g[0]) + np.abs(g[1]) > 0)
    pix = rng.choice(cand, 64, replace=False)

    def f(which, idx, delta):
        a = [x.clone() for x in args]
        a[which][idx] += delta
        return float(pr.evaluate(*a))

    for which in range(6):
        idxs = pix if which < 2 else range(args[which].numel())
        for i in idxs:
            fd = (f(which, int(i), h) - f(which, int(i), -h)) / (2 * h)
            assert abs(fd - g[which][i]) <= 1e-5 * max(1., abs(g[which][i])), (which, i)


def test_emc_nll_fp32_terms_close_to_fp64():
    size, d, ds, par, model, bg, pm, vscale = _emc_case(seed=10)
    v64, g64 = _emc_problem(size, d, par, pm, bg, vscale, 'fp64').evaluate(
        *_emc_args(model, par), grad=True)
    v32, g32 = _emc_problem(size, d, par, pm, bg, vscale, 'fp32').evaluate(
        *_emc_args(model, par), grad=True)
    assert abs(float(v32) - float(v64)) <= 1e-5 * abs(float(v64))
    for a, b in zip(g32, g64):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-3 * np.abs(b).max()


def test_emc_nll_matches_reference_likelihood():
    """At grid values the E-step NLL of each frame in its argmax state is
    minus the reference likelihood there plus the Poisson term:
    NLL = -sum_d (prob[rmax_d, d] + K_d log s_d) on the golden iterations."""
    from helpers import golden_dataset, golden_states, load_golden
    from rspi import geometry
    for name in ('case_a', 'case_b'):
        g = load_golden(name)
        ds = golden_dataset(g)
        size, num_rot = int(g['size']), int(g['num_rot'])
        sx, sy, dia, _ = golden_states(g)
        _, pm = E.generate_masks(size)
        scales = E.get_scales(ds, bool(g['need_scaling']))
        for it in (1, 2):
            model = g['model_in_%d' % it]
            rmax = g['rmax_%d' % it]
            s0, j = rmax // num_rot, rmax % num_rot
            _, vscale = E.msum_vscale(model, sx, sy, dia, size, ds['bg'], pm, E.get_powder(ds))
            par = dict(dia=dia[s0], sx=sx[s0], sy=sy[s0], scale=scales,
                       rot_cs=geometry.emc_rotation_table(num_rot).reshape(-1, 2)[j])
            from rspi.adjoint import EMCNLLProblem
            from rspi.device import DevicePhotons
            ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                               ds['count_multi'], size * size, bool(g['need_scaling']))
            pr = EMCNLLProblem(ph, size, par['rot_cs'], pm, ds['bg'], vscale, precision='fp64')
            val = float(pr.evaluate(*_emc_args(model, par)))
            kmat = E.sparse_frames(ds, pm < 1)
            k_tot = np.asarray(kmat.sum(1)).ravel()
            want = -np.sum(g['prob_%d' % it][rmax, np.arange(rmax.size)] + k_tot * np.log(scales))
            np.testing.assert_allclose(val, want, rtol=1e-11)


def test_emc_nll_autograd_function():
    from rspi.adjoint import emc_nll
    size, d, ds, par, model, bg, pm, vscale = _emc_case(seed=11)
    pr = _emc_problem(size, d, par, pm, bg, vscale, 'fp64')
    args = [a.clone().requires_grad_(True) for a in _emc_args(model, par)]
    loss = emc_nll(pr, *args)
    loss.backward()
    _, g = pr.evaluate(*_emc_args(model, par), grad=True)
    for a, b in zip(args, g):
        assert torch.allclose(a.grad, b, rtol=1e-12, atol=0)
