"""Differentiable negative log-likelihoods (row a16): the MaxLP pixel NLL
with an L-BFGS update that stands beside the pattern/grid search, and the
E-step NLL through model slicing (``EMCNLLProblem`` / ``EMCNLL``).

``NLLProblem`` fixes the data (photons, frame orientations) and evaluates

    NLL(F, dia, sx, sy, scale) = sum_d sum_t s_d |F_t + r_dt|^2 - k_dt log(s_d |F_t + r_dt|^2)

over the phaser pixels with librspi's hand-written adjoint (``rspi_nll``).
``MaxLPNLL`` wraps it as a ``torch.autograd.Function``: forward computes the
value only; backward re-runs the kernels in gradient mode (nothing frames x
pixels is stored).  ``lbfgs_update`` minimises it over the model pixels
(optionally the per-frame parameters) with ``torch.optim.LBFGS``.
"""
import numpy as np
import torch

from . import geometry
from .device import call, cur_stream, ptr

_f64 = torch.float64


class NLLProblem:
    """Fixed data of the NLL: photons, frame rotations, phaser pixels."""

    def __init__(self, photons, size, ang, precision='fp32'):
        if precision not in ('fp32', 'fp64'):
            raise ValueError('precision must be fp32 or fp64')
        self.ph = photons
        self.size = int(size)
        self.device = dev = photons.device
        self.prec = 0 if precision == 'fp32' else 1
        ang = np.asarray(ang, dtype='f8').ravel()
        if ang.size != photons.num_data:
            raise ValueError('one angle per frame is required')
        self.rot_cs = torch.from_numpy(geometry.phaser_rotation_table(ang)).to(dev)
        qx, qy, qrad, mask, _ = geometry.phaser_qvals(self.size)
        self.pixels = np.flatnonzero(mask).astype('i4')
        mask_idx = np.full(self.size ** 2, -1, dtype='i4')
        mask_idx[self.pixels] = np.arange(self.pixels.size, dtype='i4')
        t = lambda a, dt=_f64: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        self.mask_idx = t(mask_idx, torch.int32)
        self.pix_t = t(self.pixels, torch.int64)
        self.qx, self.qy, self.qrad = t(qx[self.pixels]), t(qy[self.pixels]), t(qrad[self.pixels])
        self.n_pix = int(self.pixels.size)
        self.out = torch.empty(1, dtype=_f64, device=dev)

    def evaluate(self, fre, fim, dia, sx, sy, scale, grad=False):
        """NLL (float) and, with ``grad``, the gradient tensors
        (dRe F, dIm F, d dia, d sx, d sy, d scale)."""
        n = self.ph.num_data
        c = lambda v: v.detach().to(self.device, _f64).contiguous()  # noqa: E731
        fre, fim, dia, sx, sy, scale = c(fre), c(fim), c(dia), c(sx), c(sy), c(scale)
        g = [torch.empty(self.n_pix, dtype=_f64, device=self.device) for _ in range(2)] + \
            [torch.empty(n, dtype=_f64, device=self.device) for _ in range(4)] if grad else [None] * 6
        ph = self.ph
        call('rspi_nll', self.prec, int(grad), ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum),
             ptr(ph.multi_accum), ptr(ph.place_ones), ptr(ph.place_multi), ptr(ph.count_multi),
             n, ptr(self.rot_cs), self.size, ptr(self.mask_idx), self.n_pix, ptr(fre), ptr(fim),
             ptr(self.qx), ptr(self.qy), ptr(self.qrad), ptr(dia), ptr(sx), ptr(sy), ptr(scale),
             ptr(self.out), *[ptr(x) for x in g], ptr(ph.err.t), cur_stream())
        if grad:
            return self.out.clone(), g
        return self.out.clone()

    def model_pixels(self, model):
        """(Re, Im) of a full complex model at the phaser pixels."""
        m = torch.as_tensor(np.asarray(model)).to(self.device).reshape(-1)[self.pix_t]
        return m.real.to(_f64).contiguous(), m.imag.to(_f64).contiguous()


class MaxLPNLL(torch.autograd.Function):
    """NLL with the hand-written adjoint as its backward."""

    @staticmethod
    def forward(ctx, fre, fim, dia, sx, sy, scale, problem):
        ctx.save_for_backward(fre, fim, dia, sx, sy, scale)
        ctx.problem = problem
        return problem.evaluate(fre, fim, dia, sx, sy, scale, grad=False).reshape(())

    @staticmethod
    def backward(ctx, gout):
        fre, fim, dia, sx, sy, scale = ctx.saved_tensors
        _, g = ctx.problem.evaluate(fre, fim, dia, sx, sy, scale, grad=True)
        outs = [x * gout for x in g]
        return tuple(o.to(v.dtype) for o, v in zip(outs, (fre, fim, dia, sx, sy, scale))) + (None,)


def nll(problem, fre, fim, dia, sx, sy, scale):
    return MaxLPNLL.apply(fre, fim, dia, sx, sy, scale, problem)


def lbfgs_update(problem, model, dia, sx, sy, scale, steps=50, params=False, history=20):
    """Minimise the NLL over the phaser pixels of ``model`` (complex, size^2)
    with L-BFGS; the per-frame parameters are optimised too with ``params``.
    Returns the updated full model (host complex128), the final NLL and the
    per-frame parameters."""
    fre, fim = problem.model_pixels(model)
    dev = problem.device
    p = lambda a: torch.as_tensor(np.asarray(a, dtype='f8')).to(dev).clone()  # noqa: E731
    fre.requires_grad_(True)
    fim.requires_grad_(True)
    fd, fx, fy, fs = p(dia), p(sx), p(sy), p(scale)
    var = [fre, fim] + ([fd, fx, fy, fs] if params else [])
    for v in var:
        v.requires_grad_(True)
    opt = torch.optim.LBFGS(var, lr=1, max_iter=steps, history_size=history,
                            line_search_fn='strong_wolfe')

    def closure():
        opt.zero_grad()
        loss = nll(problem, fre, fim, fd, fx, fy, fs)
        loss.backward()
        return loss

    opt.step(closure)
    with torch.no_grad():
        final = float(nll(problem, fre, fim, fd, fx, fy, fs))
    out = np.array(model, dtype=np.complex128).ravel().copy()
    out[problem.pixels] = (fre.detach() + 1j * fim.detach()).cpu().numpy()
    return out, final, (fd.detach().cpu().numpy(), fx.detach().cpu().numpy(),
                        fy.detach().cpu().numpy(), fs.detach().cpu().numpy())


# ---------------------------------------------------------------------------
# E-step side: the likelihood through model slicing (rspi_emc_nll)
# ---------------------------------------------------------------------------
class EMCNLLProblem:
    """Fixed data of the E-step NLL: photons, frame orientations, the
    likelihood pixels, background and vscale (kernels.cu:6-82,116-137)."""

    def __init__(self, photons, size, rot_cs, probmask, bg, vscale, precision='fp32'):
        if precision not in ('fp32', 'fp64'):
            raise ValueError('precision must be fp32 or fp64')
        self.ph = photons
        self.size = int(size)
        self.device = dev = photons.device
        self.prec = 0 if precision == 'fp32' else 1
        rc = torch.as_tensor(np.asarray(rot_cs, dtype='f8') if not torch.is_tensor(rot_cs)
                             else rot_cs)
        self.rot_cs = rc.to(dev, _f64).reshape(-1).contiguous()
        if self.rot_cs.numel() != 2 * photons.num_data:
            raise ValueError('one (cos, sin) pair per frame is required')
        sel, pix2sel, _ = geometry.sel_pixels(probmask)
        t = lambda a, dt=_f64: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        self.sel_pix = t(sel if sel.size else np.zeros(1, 'i4'), torch.int32)
        self.n_sel = int(sel.size)
        self.pix2sel = t(pix2sel, torch.int32)
        self.bg = t(np.asarray(bg, dtype='f8').ravel())
        self.vscale = float(vscale)
        self.out = torch.empty(1, dtype=_f64, device=dev)

    def evaluate(self, mre, mim, dia, sx, sy, scale, grad=False):
        """NLL and, with ``grad``, (dRe M, dIm M, d dia, d sx, d sy, d scale)."""
        n, npix = self.ph.num_data, self.size ** 2
        c = lambda v: v.detach().to(self.device, _f64).contiguous()  # noqa: E731
        model = torch.complex(c(mre), c(mim)).contiguous()
        dia, sx, sy, scale = c(dia), c(sx), c(sy), c(scale)
        g = ([torch.empty(npix, dtype=_f64, device=self.device) for _ in range(2)] +
             [torch.empty(n, dtype=_f64, device=self.device) for _ in range(4)]) if grad \
            else [None] * 6
        ph = self.ph
        call('rspi_emc_nll', self.prec, int(grad), ptr(model), self.size, ptr(self.bg),
             ptr(self.sel_pix), self.n_sel, ptr(self.pix2sel), ptr(ph.ones), ptr(ph.multi),
             ptr(ph.ones_accum), ptr(ph.multi_accum), ptr(ph.place_ones), ptr(ph.place_multi),
             ptr(ph.count_multi), n, ptr(self.rot_cs), ptr(dia), ptr(sx), ptr(sy), ptr(scale),
             self.vscale, ptr(self.out), *[ptr(x) for x in g], ptr(ph.err.t), cur_stream())
        if grad:
            return self.out.clone(), g
        return self.out.clone()


class EMCNLL(torch.autograd.Function):
    """E-step NLL with the hand-written adjoint as its backward (the slices
    are recomputed in backward; nothing frames x states is kept)."""

    @staticmethod
    def forward(ctx, mre, mim, dia, sx, sy, scale, problem):
        ctx.save_for_backward(mre, mim, dia, sx, sy, scale)
        ctx.problem = problem
        return problem.evaluate(mre, mim, dia, sx, sy, scale, grad=False).reshape(())

    @staticmethod
    def backward(ctx, gout):
        mre, mim, dia, sx, sy, scale = ctx.saved_tensors
        _, g = ctx.problem.evaluate(mre, mim, dia, sx, sy, scale, grad=True)
        outs = [x * gout for x in g]
        return tuple(o.to(v.dtype) for o, v in zip(outs, (mre, mim, dia, sx, sy, scale))) + (None,)


def emc_nll(problem, mre, mim, dia, sx, sy, scale):
    return EMCNLL.apply(mre, mim, dia, sx, sy, scale, problem)
