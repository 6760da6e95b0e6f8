"""FP64 NumPy/SciPy oracle for the MaxLP model refinement (ER and difference
map, the step after the pattern search).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows maxLP.py:32-33,71-75 (the inverse data mask ``minvmask`` from the
integer-centred radius ``mrad``), 271-275 (``proj_fourier``), 277-281
(``proj_real``), 283-290 (``er``, ``diffmap``), 292-298 (``_get_support``)
and 342-354 (``_improve_model``).  The reference transforms with NumPy's
``fftshift(fftn(ifftshift(.)))`` convention and filters the support with
``cupyx.scipy.ndimage.gaussian_filter`` (sigma 3, 'reflect' edges, radius
12); SciPy's ``ndimage.gaussian_filter`` is the same algorithm on the host.
Arrays are flat complex128 of ``size * size`` pixels (row-major).
"""
import numpy as np
from scipy import ndimage, special


def mrad(size):
    """Integer-centred pixel radius of every model pixel, maxLP.py:28-31."""
    x, y = np.indices((size, size), dtype='f8')
    x = x.ravel() - size // 2
    y = y.ravel() - size // 2
    return np.sqrt(x ** 2 + y ** 2)


def get_invmask(size, r=4):
    """Pixels the Fourier projection takes from the data: r <= mrad <
    size//2, maxLP.py:71-75."""
    m = np.ones(size ** 2, dtype=bool)
    rad = mrad(size)
    m[rad < r] = False
    m[rad >= size // 2] = False
    return m


def centered_ifft(x, size):
    return np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(x.reshape(size, size))))


def centered_fft(x, size):
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x.reshape(size, size))))


def proj_fourier(fconv, x, minvmask):
    """maxLP.py:271-274: x with the data pixels replaced by fconv's."""
    out = x.copy()
    out[minvmask] = fconv[minvmask]
    return out


def proj_real(x, minvsuppmask, size):
    """maxLP.py:276-280: real part of the centred inverse transform, negative
    values and pixels outside the support set to 0, transformed back."""
    rmodel = np.real(centered_ifft(x, size))
    rmodel[rmodel < 0] = 0
    rmodel[minvsuppmask.reshape(size, size)] = 0
    return centered_fft(rmodel, size).ravel()


def er(fconv, x, minvmask, minvsuppmask, size):
    """maxLP.py:282-284."""
    return proj_real(proj_fourier(fconv, x, minvmask), minvsuppmask, size)


def diffmap(fconv, x, minvmask, minvsuppmask, size):
    """maxLP.py:286-289."""
    p1 = proj_fourier(fconv, x, minvmask)
    return x + proj_real(2 * p1 - x, minvsuppmask, size) - p1


def support_field(fconv, size):
    """The filtered real-space amplitude the support is thresholded on,
    maxLP.py:292-295: fconv tapered by expit((mrad - 12) / 2), centred
    inverse transform, |real part| smoothed with a sigma-3 Gaussian."""
    smask = special.expit((mrad(size).reshape(size, size) - 12) * 0.5)
    rsupp = np.real(centered_ifft(fconv.reshape(size, size) * smask, size))
    return ndimage.gaussian_filter(np.abs(rsupp), 3)


def get_support(fconv, size, threshold=1.2e-4):
    """maxLP.py:292-298: True outside the support (``minvsuppmask``)."""
    return ~(support_field(fconv, size) > threshold).ravel()


def improve_model(fconv, size, minvmask=None, n_dm=10, n_er=5):
    """maxLP.py:342-354 with update_masks=True: the support from fconv, then
    n_dm difference-map and n_er error-reduction iterations from fconv.
    Returns (model, minvsuppmask)."""
    if minvmask is None:
        minvmask = get_invmask(size)
    supp = get_support(fconv, size)
    fout = fconv.copy()
    for _ in range(n_dm):
        fout = diffmap(fconv, fout, minvmask, supp, size)
    for _ in range(n_er):
        fout = er(fconv, fout, minvmask, supp, size)
    return fout, supp
