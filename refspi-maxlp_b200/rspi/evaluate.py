"""Model-update comparison on one E-step assignment: the MaxLP pattern
search (maxLP.py:304-340), the polar grid search of the NLL and the L-BFGS
update of the NLL through the hand-written adjoint (row a16), compared on
the final NLL and on the Fourier ring correlation (FRC) with the true
object transform.

Every update starts from the same model and the same frame parameters (the
E-step argmax: (shift, diameter) state and rotation per frame).  The NLL's
per-frame scale is ``rho * scale_d``: the MaxLP global rescale of the
pattern search (maxLP.py:329) times the frame's photon-count scale.
"""
import numpy as np
import torch

from . import geometry
from .adjoint import NLLProblem, lbfgs_update
from .device import MStep

_f64 = torch.float64


def frc(a, b, size, pixels=None):
    """Ring-wise correlation of two complex (size^2) transforms over integer
    pixel radii: Re sum(a conj b) / sqrt(sum |a|^2 sum |b|^2) per ring.
    ``pixels`` restricts the sums.  Returns (radii, frc) for rings with
    pixels."""
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    x = np.arange(size) - size // 2
    rad = np.rint(np.sqrt(x[:, None] ** 2 + x[None, :] ** 2)).astype(int).ravel()
    sel = np.zeros(size * size, bool)
    if pixels is None:
        sel[:] = True
    else:
        sel[np.asarray(pixels)] = True
    r = rad[sel]
    num = np.bincount(r, weights=(a[sel] * np.conj(b[sel])).real)
    na = np.bincount(r, weights=np.abs(a[sel]) ** 2)
    nb = np.bincount(r, weights=np.abs(b[sel]) ** 2)
    ok = (na > 0) & (nb > 0)
    radii = np.flatnonzero(ok)
    return radii, num[ok] / np.sqrt(na[ok] * nb[ok])


def compare_updates(photons, size, model, truth, rmax, num_rot, state_values, n_phase=64,
                    n_amp=32, lbfgs_steps=50, num_iter=10):
    """Run the three updates from ``model`` and report NLL and FRC.

    ``rmax`` (device int32, one per frame) gives each frame's state
    ``s*num_rot + j``; ``state_values`` (S0 x 3 device FP64) the (sx, sy,
    dia) of each state.  Returns a dict with the models, NLLs and FRCs."""
    dev = photons.device
    n = photons.num_data
    n_ref = int(state_values.shape[0])
    ms = MStep(photons, size, num_iter)
    rot = torch.from_numpy(geometry.phaser_rotation_table(
        np.arange(num_rot) * np.pi / num_rot)).to(dev)
    ms.frame_params_from_rmax(rmax, num_rot, n_ref)
    start = np.asarray(model, dtype=np.complex128).ravel()

    f_pat = torch.from_numpy(start.copy()).to(dev)
    ms.run(f_pat, state_values, rot)
    rho = float(ms.rescale[0].item())
    scale = photons.scales * rho

    f_grid = torch.from_numpy(start.copy()).to(dev)
    ms.grid(f_grid, state_values, rot, scale, n_phase, n_amp)

    fstate = ms.fstate.long()
    vals = state_values[fstate]
    ang = (ms.frot.double() * np.pi / num_rot).cpu().numpy()
    sx, sy, dia = vals[:, 0], vals[:, 1], vals[:, 2]
    prob = NLLProblem(photons, size, ang, precision='fp64')
    photons.err.check('model-update comparison')

    def nll_of(m):
        fre, fim = prob.model_pixels(m)
        return float(prob.evaluate(fre, fim, dia, sx, sy, scale))

    s_np = scale.cpu().numpy()
    d_np, x_np, y_np = dia.cpu().numpy(), sx.cpu().numpy(), sy.cpu().numpy()
    m_lb, nll_lb, _ = lbfgs_update(prob, start, d_np, x_np, y_np, s_np, steps=lbfgs_steps)
    m_grid = f_grid.cpu().numpy()
    m_glb, nll_glb, _ = lbfgs_update(prob, m_grid, d_np, x_np, y_np, s_np, steps=lbfgs_steps)
    models = {'start': start, 'pattern': f_pat.cpu().numpy(), 'grid': m_grid,
              'lbfgs': m_lb, 'grid_lbfgs': m_glb}
    out = {'rescale': rho, 'n_frames': n, 'pixels': int(prob.n_pix),
           'nll': {k: nll_of(v) for k, v in models.items()}, 'frc': {}, 'frc_mean': {}}
    if truth is not None:
        for k, v in models.items():
            radii, f = frc(v, truth, size, prob.pixels)
            out['frc'][k] = f.tolist()
            out['frc_mean'][k] = float(f.mean())
        out['frc_radii'] = radii.tolist()
    out['models'] = models
    return out
