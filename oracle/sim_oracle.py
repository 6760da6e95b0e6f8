"""FP64 NumPy restatement of the reference's data simulator (make_data.py).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the checker for the
CUDA simulator, never part of it.

Covered, in the reference's order of operations:

* the deterministic object of ``make_obj`` (``create_random = no``,
  make_data.py:95-138): 55 parabolic discs, and for a heterogeneous object
  25 "wobble" discs, at centres and radii that are functions of the disc
  index;
* the frame's model of each object type (make_data.py:294-309):
  ``iso`` the object's transform, ``homo``/``mix``/``blur`` that plus the
  wobble sub-unit's transform with a phase ramp (``mix`` alternating between
  two ramps by frame parity, one of them mirrored left-right);
* the expected photon counts of one frame (make_data.py:310-322): the
  holographic intensity of that model with the frame's sphere shift,
  diameter, ``rel_scale`` and fluence scale, times the detector mask,
  normalised to ``mean_count`` photons, rotated by the frame's angle with
  bilinear interpolation, plus the background;
* the sparse lists of a frame of counts (make_data.py:323-328).

The random draws (object discs with ``create_random``, the per-frame
parameters and the Poisson counts) come from unseeded generators in the
reference; they are checked statistically, not value by value.
"""
import numpy as np

from . import emc_oracle as E


def _disc(acc, x, y, c0, c1, rad):
    """acc += 1 - (r / rad)^2 on the pixels with r <= rad (make_data.py:104-105)."""
    r = np.sqrt((x - c0) ** 2 + (y - c1) ** 2)
    inside = r <= rad
    acc[inside] += 1. - (r[inside] / rad) ** 2


def deterministic_object(size, hetro=False):
    """``make_obj`` with ``create_random = no`` (make_data.py:95-138).
    Returns (object, wobble object or None), (size, size) float64."""
    mcen = size // 2
    x, y = np.indices((size, size), dtype='f8')
    obj = np.zeros((size, size))
    for i in range(55):
        rad = (0.7 + 0.3 * (np.cos(2.5 * i) - np.sin(i / 4))) * size / 20.
        cen0 = (3 * np.sin(2 * i) + 0.5 * np.sin(i / 2)) * size / 45. + mcen * 4. / 4.4
        cen1 = (0.5 * np.cos(i / 2) + 3 * np.cos(i / 2)) * size / 45. + mcen * 4. / 4.4
        if not float(np.sqrt((cen0 - mcen) ** 2 + (cen1 - mcen) ** 2) + rad) < mcen:
            raise ValueError('disc %d leaves the detector' % i)
        _disc(obj, x, y, cen0, cen1, rad)
    if not hetro:
        return obj, None
    wob = np.zeros((size, size))
    for i in range(25):
        rad = (0.7 + 0.3 * (np.sin(i) - np.cos(i / 2))) * size / 30.
        cen0 = (np.sin(2 * i) - 3 * np.cos(i)) * size / 60. + mcen * 4.6 / 7.
        cen1 = (np.cos(i) - np.sin(i / 2)) * size / 60. + mcen * 4.6 / 7.
        if not float(np.sqrt((cen0 - mcen) ** 2 + (cen1 - mcen) ** 2) + rad) < mcen:
            raise ValueError('wobble disc %d leaves the detector' % i)
        _disc(wob, x, y, cen0, cen1, rad)
    return obj, wob


def centred_fft(obj):
    """fftshift(fftn(ifftshift(obj))) (make_data.py:282-284)."""
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(obj)))


def qvals(size):
    """qx, qy = (index - size//2) / (2 (size//2)) (make_data.py:290-291)."""
    x, y = np.indices((size, size), dtype='f8')
    mcen = size // 2.
    return (x - mcen) / (2 * mcen), (y - mcen) / (2 * mcen)


def frame_model(kind, model, wobble_model, i, w, size):
    """The frame's Fourier model (make_data.py:294-309); ``w`` is the frame's
    wobble amplitude (4.5 for ``homo`` and ``mix``, make_data.py:296,300)."""
    if kind == 'iso':
        return model
    qx, qy = qvals(size)
    if kind == 'homo':
        a = np.fliplr(wobble_model * np.exp(2 * np.pi * 1j * (qx * w + (-3.7) * qy * w)))
        b = wobble_model * np.exp(2 * np.pi * 1j * (qx * w + qy * w))
        return model + (a + b) / 2
    if kind == 'mix':
        if i % 2 == 0:
            return model + wobble_model * np.exp(2 * np.pi * 1j * (qx * w + qy * w))
        return model + np.fliplr(wobble_model *
                                 np.exp(2 * np.pi * 1j * (qx * w + (-3.7) * qy * w)))
    if kind == 'blur':
        return model + wobble_model * np.exp(2 * np.pi * 1j * (qx * w + (-3.7) * qy * w))
    raise ValueError(kind)


def detector_mask(size):
    """1 except r < 4 and r >= size//2 (make_data.py:210-216)."""
    x, y = np.indices((size, size), dtype='f8')
    cen = size // 2
    r = np.sqrt((x - cen) ** 2 + (y - cen) ** 2)
    m = np.ones((size, size))
    m[r < 4] = 0
    m[r >= cen] = 0
    return m


def expected_frame(fmodel, shiftx, shifty, dia, rel_scale, scale, angle, size, mean_count,
                   bg=None, hetro=False):
    """Expected counts of one frame (make_data.py:310-322): holographic
    intensity (no background), times the mask (twice the mask for a
    heterogeneous object), scaled to mean_count photons, rotated by
    ``angle`` (bilinear; pixels whose footprint leaves the detector are 0),
    plus ``bg`` on the others."""
    zero = np.zeros(size * size)
    view = E.holo_slice(fmodel, shiftx, shifty, dia, rel_scale, scale, size, zero)
    m = detector_mask(size).ravel()
    view = view * ((m + m) if hetro else m)
    view = view * (mean_count / view.sum())
    bgv = zero if bg is None else np.asarray(bg, dtype='f8').ravel()
    return E.rotate_slice(view, angle, 1., size, bgv, 0)


def sparse_lists(frames):
    """place_ones / place_multi / count_multi / ones / multi of dense counts
    (N, P), pixels ascending (make_data.py:323-328)."""
    f = np.asarray(frames)
    out = dict(ones=(f == 1).sum(1).astype('i4'), multi=(f > 1).sum(1).astype('i4'))
    po, pm, cm = [], [], []
    for row in f:
        po.append(np.flatnonzero(row == 1))
        many = np.flatnonzero(row > 1)
        pm.append(many)
        cm.append(row[many])
    cat = lambda a: np.concatenate(a).astype('i4') if a else np.zeros(0, 'i4')  # noqa: E731
    out.update(place_ones=cat(po), place_multi=cat(pm), count_multi=cat(cm))
    return out
