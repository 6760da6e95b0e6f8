"""FP64 NumPy oracle for the MaxLP M-step (rows a11-a14 of the hot path).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows maxLP.py:45-48 (pattern), 79-95 (q grids and masks), 107-114
(pixel constants), 154-197 (pattern search and per-candidate
log-likelihood), 216-228 (rescale), 238-258 (reference form factor, photons
of a pixel, rotations) and 304-340 (``_run_phaser``).  Written in the literal
dense form of the reference (every frame, every candidate), which is what the
CUDA kernels' sparse/analytic form is checked against.

Rotation of a model pixel into each frame (maxLP.py:250-252) is evaluated as
``x' = c*qx + (-s)*qy``, ``y' = s*qx + c*qy`` with ``c = cos(-ang)``,
``s = sin(-ang)`` -- two products and one sum, no fused multiply-add -- then
``rint(x'*size + size//2)``.  The CUDA kernel uses the same operations with
the same host-computed cos/sin table, so the photon indices are bit-exact.
"""
import numpy as np

from . import emc_oracle


def gen_pattern(nmax=8):
    """33x33 candidate offsets ``(x + iy)``, maxLP.py:45-48."""
    ind = np.arange(-nmax, nmax + 0.5, 0.5)
    x, y = np.meshgrid(ind, ind, indexing='ij')
    return (x + 1j * y).ravel()


def get_qvals(size):
    """q grids, radius and the two masks used by the phaser, maxLP.py:79-95."""
    ind = (np.arange(size, dtype='f8') - size // 2) / size
    qx, qy = np.meshgrid(ind, ind, indexing='ij')
    qx, qy = qx.ravel(), qy.ravel()
    qrad = np.sqrt(qx * qx + qy * qy)
    qrad[qrad == 0] = 1.e-6
    mask = (qrad > 4 / size) & (qrad < 0.5)
    rmask = (qrad > 0.39) & (qrad < 0.41)
    return qx, qy, qrad, mask, rmask


def rotation_table(ang):
    """``(cos(-ang), sin(-ang))`` per frame (maxLP.py:255-258 with -ang)."""
    a = -np.asarray(ang, dtype='f8')
    return np.cos(a), np.sin(a)


def photon_pixels(ang, t, size, qx, qy):
    """Detector pixel of model pixel ``t`` in every frame, maxLP.py:250-252.

    Returns the flat column index ``x*size + y`` (int64); it can fall outside
    ``[0, size^2)`` only for even sizes, where the CSR lookup reads 0.
    """
    c, s = rotation_table(ang)
    xr = c * qx[t] + (-s) * qy[t]
    yr = s * qx[t] + c * qy[t]
    x = np.rint(xr * size + size // 2).astype('i4')
    y = np.rint(yr * size + size // 2).astype('i4')
    return x.astype(np.int64) * size + y


def photons_pixel(kmat, ang, t, size, qx, qy):
    """``k_d`` of model pixel t for every frame, maxLP.py:245-253 (CSR lookup
    with summed duplicates; out-of-range columns read 0)."""
    cols = photon_pixels(ang, t, size, qx, qy)
    n, p = kmat.shape
    ok = (cols >= 0) & (cols < p)
    out = np.zeros(n)
    rows = np.arange(n)[ok]
    out[ok] = np.asarray(kmat[rows, cols[ok]]).ravel()
    return out


def fref_pixel(t, qx, qy, qrad, diams, shifts):
    """Reference-sphere amplitude of every frame at pixel t, maxLP.py:238-243."""
    sval = np.pi * qrad[t] * diams
    fref = (np.sin(sval) - sval * np.cos(sval)) / sval ** 3
    theta = 2 * np.pi * (qx[t] * shifts[:, 0] + qy[t] * shifts[:, 1])
    return fref * (np.cos(theta) + 1j * np.sin(theta))


def rescale_pixel(f_c, k_d, fref_d):
    """Per-candidate rescale ``mean(k)/mean_d|f_c + fref_d|^2``, maxLP.py:216-228."""
    f_dt = fref_d[:, None] + np.atleast_1d(f_c)[None, :]
    return k_d.mean() / (np.abs(f_dt) ** 2).mean(0)


def logq_pixel(f_c, k_d, fref_d, rescale=None):
    """Per-candidate log-likelihood, maxLP.py:181-197:
    ``mean_d(k_d log w) - mean_d(w)``, ``w = rescale*|f_c + fref_d|^2``."""
    f_c = np.atleast_1d(f_c)
    if rescale is None:
        rescale = rescale_pixel(f_c, k_d, fref_d)
    f_dt = fref_d[:, None] + f_c[None, :]
    w_dt = rescale * np.abs(f_dt) ** 2
    with np.errstate(divide='ignore', invalid='ignore'):
        return (k_d[:, None] * np.log(w_dt)).mean(0) - w_dt.mean(0)


def _argmax_nan_first(vals):
    """NumPy argmax semantics: first maximum, and a NaN counts as maximum."""
    return int(np.argmax(vals))


def run_pixel_pattern(f_t, k_d, fref_d, pattern, rescale=None, num_iter=10,
                      trace=None):
    """Pattern search of one model pixel, maxLP.py:154-179.

    Starting step ``|f|/4``; each iteration takes the best of the 1089
    candidates ``f + pattern*step`` (first index on ties); hitting the centre
    candidate divides the step by ``sqrt(1089)/5``.  When the new step is
    below ``1e-3*|f_new|`` the loop stops and returns the value *before*
    that last move (maxLP.py:162-165).
    """
    f_t = complex(f_t)
    step = abs(f_t) / 4.
    centre = pattern.size // 2
    shrink = pattern.size ** 0.5 / 5
    for _ in range(num_iter):
        cand = f_t + pattern * step
        vals = logq_pixel(cand, k_d, fref_d, rescale)
        imax = _argmax_nan_first(vals)
        f_new = f_t + pattern[imax] * step
        step_new = step / shrink if imax == centre else step
        if trace is not None:
            trace.append(imax)
        with np.errstate(divide='ignore', invalid='ignore'):
            if step_new / abs(f_new) < 1.e-3:
                break
        f_t, step = f_new, step_new
    return f_t


def run_phaser(model, kmat, sx_vals, sy_vals, dia_vals, ang_vals, size,
               pixels=None, ring_only=False, return_rescale=False):
    """``_run_phaser`` (maxLP.py:304-340): ring pass with per-candidate
    rescale, global rescale = mean over the ring, then the main pass over
    ``mask`` with that rescale.  ``pixels`` restricts the main pass (for
    bounded CPU timing); the ring pass always runs in full.
    """
    qx, qy, qrad, mask, rmask = get_qvals(size)
    pattern = gen_pattern(8)
    shifts = np.array([sx_vals, sy_vals]).T
    diams = np.asarray(dia_vals, dtype='f8')
    fconv = np.array(model, dtype=np.complex128).ravel().copy()

    def consts(t):
        return (photons_pixel(kmat, ang_vals, t, size, qx, qy),
                fref_pixel(t, qx, qy, qrad, diams, shifts))

    ring = np.where(rmask)[0]
    for t in ring:
        k_d, fref_d = consts(t)
        fconv[t] = run_pixel_pattern(fconv[t], k_d, fref_d, pattern, None, 10)
    rescales = np.zeros(size ** 2)
    for t in ring:
        k_d, fref_d = consts(t)
        rescales[t] = rescale_pixel(fconv[t], k_d, fref_d)[0]
    rescale = np.mean(rescales[rmask])
    if not ring_only:
        main = np.where(mask)[0] if pixels is None else np.asarray(pixels)
        for t in main:
            k_d, fref_d = consts(t)
            fconv[t] = run_pixel_pattern(fconv[t], k_d, fref_d, pattern, rescale, 10)
    if return_rescale:
        return fconv, rescale
    return fconv
