"""Hand-written adjoint of the MaxLP negative log-likelihood (row a16).

Checked against (1) torch autograd through the FP64 dense restatement in
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
