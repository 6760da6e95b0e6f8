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

The E-step side (``emc_nll_torch``): minus the reference likelihood
calc_prob_all (emc.py:194-199, kernels.cu:116-137) of each frame in its
chosen orientation, differentiable in the complex model and the continuous
diameter, shift and scale, with the Poisson term K_d log s_d that the
reference drops (constant over states) kept.
"""
import numpy as np
import torch

from . import emc_oracle as E
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


# ---------------------------------------------------------------------------
# EMC side: the likelihood through model slicing (kernels.cu:6-82,116-137)
# ---------------------------------------------------------------------------
def emc_nll_torch(m_re, m_im, dia, sx, sy, scale, vscale, kmat, angles, size, bg, sel):
    """Dense FP64 EMC negative log-likelihood, differentiable in torch:

        NLL = sum_d [ vscale s_d sum_{q in sel} W_d(q)
                      - sum_{p in sel} K_d(p) (log s_d + L_d(p)) ]

    W_d = |M + ff(pi rho dia_d / size) e^{2 pi i ((x-c) sx_d + (y-c) sy_d)/size}|^2 + bg
    (holo_slice, kernels.cu:58-75) and L_d the bilinear rotated log-slice of
    W_d plus bg (rotate_slice with log_flag, kernels.cu:19-41; -1000 where
    invalid, a constant).  ``m_*`` (P,), the per-frame parameters (N,),
    ``kmat`` a scipy CSR (N, P) of photons, ``angles`` (N,) fixed, ``sel``
    (P,) bool.  The bilinear indices and weights depend on the fixed angles
    only."""
    size = int(size)
    x, y = np.indices((size, size), dtype='f8')
    cen = np.floor(size / 2.)
    dx = torch.tensor((x - cen).ravel())
    dy = torch.tensor((y - cen).ravel())
    rho = torch.sqrt(dx * dx + dy * dy)
    bg_t = torch.tensor(np.asarray(bg, dtype='f8').ravel())
    sel_t = torch.tensor(np.asarray(sel, dtype=bool).ravel())
    s = rho[None, :] * np.pi * dia[:, None] / size
    s = torch.where(s == 0., torch.full_like(s, 1.e-5), s)
    ff = (torch.sin(s) - s * torch.cos(s)) / (s * s * s)
    ph = 2. * np.pi * (dx[None, :] * sx[:, None] + dy[None, :] * sy[:, None]) / size
    zr = torch.cos(ph) * ff + m_re[None, :]
    zi = torch.sin(ph) * ff + m_im[None, :]
    w = zr * zr + zi * zi + bg_t[None, :]                          # (N, P)
    total = (vscale * scale * w[:, sel_t].sum(1)).sum()
    for d in range(w.shape[0]):
        row = kmat.getrow(d)
        pix = row.indices[np.asarray(sel, dtype=bool).ravel()[row.indices]]
        k = torch.tensor(np.asarray(kmat[d, pix].toarray()).ravel() if pix.size else np.zeros(0))
        if pix.size == 0:
            continue
        ix, iy, fx, fy, valid = E.rotation_geometry(float(angles[d]), size)
        ix, iy, fx, fy, valid = ix[pix], iy[pix], fx[pix], fy[pix], valid[pix]
        ixc, iyc = np.where(valid, ix, 0), np.where(valid, iy, 0)
        cx, cy = 1. - fx, 1. - fy
        wd = w[d]
        b = (wd[torch.tensor(ixc * size + iyc)] * torch.tensor(cx * cy) +
             wd[torch.tensor((ixc + 1) * size + iyc)] * torch.tensor(fx * cy) +
             wd[torch.tensor(ixc * size + iyc + 1)] * torch.tensor(cx * fy) +
             wd[torch.tensor((ixc + 1) * size + iyc + 1)] * torch.tensor(fx * fy))
        b = b + bg_t[torch.tensor(pix)]
        ok = torch.tensor(valid) & (b >= 1.e-20)
        logv = torch.where(ok, torch.log(torch.where(ok, b, torch.ones_like(b))),
                           torch.full_like(b, E.LOG_SENTINEL))
        total = total - (k * (torch.log(scale[d]) + logv)).sum()
    return total


def emc_nll_and_grad(model, dia, sx, sy, scale, vscale, kmat, angles, size, bg, sel):
    """EMC NLL and its gradient (dM as d/dRe + i d/dIm over every pixel;
    per-frame d/ddia, d/dsx, d/dsy, d/dscale) in FP64 via torch.autograd."""
    t = lambda a: torch.tensor(np.asarray(a, dtype=np.float64), requires_grad=True)  # noqa: E731
    model = np.asarray(model, dtype=np.complex128).ravel()
    mr, mi = t(model.real), t(model.imag)
    dd, xx, yy, ss = t(dia), t(sx), t(sy), t(scale)
    loss = emc_nll_torch(mr, mi, dd, xx, yy, ss, float(vscale), kmat, angles, size, bg, sel)
    loss.backward()
    g = lambda v: v.grad.numpy().copy()  # noqa: E731
    return float(loss.detach()), g(mr) + 1j * g(mi), g(dd), g(xx), g(yy), g(ss)
