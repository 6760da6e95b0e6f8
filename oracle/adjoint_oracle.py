"""FP64 reference for the differentiable MaxLP negative log-likelihood (a16).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference has no gradient: ``get_grad_pixel`` (maxLP.py:199-214) is
broken (it uses an undefined ``f_d``) but shows the intended objective, the
MaxLP per-pixel log-likelihood of maxLP.py:181-197.  The build defines its
continuous generalisation over every phaser pixel t and frame d:

    NLL = sum_d sum_t [ s_d |F_t + r_dt|^2 - k_dt log(s_d |F_t + r_dt|^2) ]

with r_dt = ff(pi q_t dia_d) exp(2 pi i (qx_t sx_d + qy_t sy_d))
(maxLP.py:238-243), k_dt the photons of frame d at model pixel t's rotated
detector pixel (maxLP.py:245-253, fixed orientations) and s_d the per-frame
scale.  With s_d = rescale for every frame this is -N * sum_t Q_t of
maxLP.py:197 (up to the frame-independent k log(rescale) terms).

``nll_torch`` evaluates it densely in torch FP64 so that torch.autograd
gives the reference gradient; ``photon_matrix`` builds k_dt with the
oracle's exact rotation (maxlp_oracle.photon_pixels).
"""
import numpy as np
import torch

from . import maxlp_oracle as M


def photon_matrix(kmat, ang, size, pixels):
    """k[d, i] = photons of frame d at the detector pixel of model pixel
    pixels[i] (dense, FP64)."""
    qx, qy, _, _, _ = M.get_qvals(size)
    return np.stack([M.photons_pixel(kmat, ang, int(t), size, qx, qy) for t in pixels], axis=1)


def nll_torch(f_re, f_im, dia, sx, sy, scale, k, qx, qy, qrad):
    """Dense FP64 NLL; every argument a torch tensor.  f_* over the pixels
    (P,), the per-frame parameters (N,), k (N, P), q* (P,)."""
    x = np.pi * qrad[None, :] * dia[:, None]
    ff = (torch.sin(x) - x * torch.cos(x)) / x ** 3
    th = 2 * np.pi * (qx[None, :] * sx[:, None] + qy[None, :] * sy[:, None])
    zr = f_re[None, :] + ff * torch.cos(th)
    zi = f_im[None, :] + ff * torch.sin(th)
    a = zr * zr + zi * zi
    w = scale[:, None] * a
    return (w - k * torch.log(w)).sum()


def nll_and_grad(f, dia, sx, sy, scale, k, size, pixels):
    """NLL and its gradient (dF as complex d/dRe + i d/dIm; per-frame
    d/ddia, d/dsx, d/dsy, d/dscale) in FP64 via torch.autograd."""
    _, _, qrad, _, _ = M.get_qvals(size)
    qx, qy, _, _, _ = M.get_qvals(size)
    t = lambda a: torch.tensor(np.asarray(a, dtype=np.float64), requires_grad=True)  # noqa: E731
    f = np.asarray(f, dtype=np.complex128)
    fr, fi = t(f.real), t(f.imag)
    dd, xx, yy, ss = t(dia), t(sx), t(sy), t(scale)
    pix = np.asarray(pixels)
    loss = nll_torch(fr, fi, dd, xx, yy, ss, torch.tensor(k, dtype=torch.float64),
                     torch.tensor(qx[pix]), torch.tensor(qy[pix]), torch.tensor(qrad[pix]))
    loss.backward()
    g = lambda v: v.grad.numpy().copy()  # noqa: E731
    return float(loss.detach()), g(fr) + 1j * g(fi), g(dd), g(xx), g(yy), g(ss)


def grid_pixel(k_d, fref_d, s_d, n_phase=64, n_amp=32):
    """Polar grid search of one pixel's NLL (frame by frame, FP64):
    NLL(F) = sum_d s_d |F + r_d|^2 - k_d log |F + r_d|^2 over
    F = a_j e^{i phi_i}, phi_i = 2 pi i / n_phase, a_j = A (j + 1) / n_amp,
    A = sqrt(sum k / sum s) + max_d |r_d|; the lowest value, first index on
    ties (candidate index i * n_amp + j).  Returns (F, NLL, index)."""
    k_d = np.asarray(k_d, dtype=np.float64)
    s_d = np.asarray(s_d, dtype=np.float64)
    amp = np.sqrt(k_d.sum() / s_d.sum()) + np.abs(fref_d).max()
    i = np.arange(n_phase)[:, None]
    j = np.arange(n_amp)[None, :]
    a = amp * (j + 1) / n_amp
    ph = 2 * np.pi * i / n_phase
    cand = (a * np.cos(ph) + 1j * a * np.sin(ph)).ravel()
    z = cand[None, :] + fref_d[:, None]
    w = np.abs(z) ** 2
    with np.errstate(divide='ignore'):
        nll = (s_d[:, None] * w).sum(0) - (k_d[:, None] * np.log(w)).sum(0)
    idx = int(np.argmin(nll))
    return cand[idx], nll[idx], idx
