"""Static geometry computed once per reconstructor (host, NumPy).

These are the reference constructor's own set-up computations -- state
grids, masks, q grids and the angle tables -- evaluated on the host exactly
as the reference evaluates them, so that every integer derived from them
(mask membership, pixel lists, state tables) is identical.  Nothing here is
per-iteration work.
"""
import numpy as np


def parse_triple(text):
    """``"lo hi n"`` -> (lo, hi, n) floats, emc.py:68-70."""
    vals = tuple(float(s) for s in str(text).split())
    if len(vals) != 3:
        raise ValueError('expected "lo hi n", got %r' % (text,))
    return vals


def state_grid(sx, sy, dia):
    """Flattened meshgrid of (shiftx, shifty, sphere_dia), emc.py:71-78."""
    gx, gy, gd = np.meshgrid(np.linspace(sx[0], sx[1], int(sx[2])),
                             np.linspace(sy[0], sy[1], int(sy[2])),
                             np.linspace(dia[0], dia[1], int(dia[2])), indexing='ij')
    num_states = np.array([sx[-1], sy[-1], dia[-1]]).astype('i4')
    return gx.ravel(), gy.ravel(), gd.ravel(), num_states


def state_values(shiftx, shifty, sphere_dia, num_states):
    """(n_states0, 3) table of the values ``_unravel_rmax`` reports for each
    state: ``unique(grid)[index]`` (emc.py:219-222).  For increasing grids this
    is the grid itself; a decreasing grid is reported sorted, as the
    reference does."""
    n0 = int(np.prod(num_states))
    isx, isy, idia = np.unravel_index(np.arange(n0), tuple(int(v) for v in num_states))
    ux, uy, ud = np.unique(shiftx), np.unique(shifty), np.unique(sphere_dia)
    if isx.max() >= ux.size or isy.max() >= uy.size or idia.max() >= ud.size:
        raise ValueError('state grid has repeated values; unique() cannot index it '
                         '(emc.py:220-222)')
    return np.ascontiguousarray(np.stack([ux[isx], uy[isy], ud[idia]], axis=1))


def detector_radius(size):
    """Integer-centred radius of every pixel, emc.py:81-84."""
    x, y = np.indices((size, size), dtype='f8')
    x = x.ravel() - size // 2
    y = y.ravel() - size // 2
    return x, y, np.sqrt(x * x + y * y)


def emc_masks(size):
    """``invmask`` and ``probmask``, emc.py:89-98."""
    _, _, rad = detector_radius(size)
    invmask = np.zeros(size ** 2, dtype=bool)
    invmask[rad < 4] = True
    invmask[rad >= size // 2] = True
    probmask = np.zeros(size ** 2, dtype='i4')
    probmask[rad >= size // 2] = 2
    probmask[rad < size // 8] = 1
    probmask[rad < 4] = 2
    return invmask, probmask


def sel_pixels(probmask):
    """Likelihood pixels (probmask < 1, kernels.cu:129) in pixel order, the
    pixel -> sel index map (-1 elsewhere) and the padded row length."""
    sel = np.flatnonzero(probmask < 1).astype('i4')
    pix2sel = np.full(probmask.size, -1, dtype='i4')
    pix2sel[sel] = np.arange(sel.size, dtype='i4')
    p_pad = max(32, -(-sel.size // 32) * 32)
    return sel, pix2sel, p_pad


def emc_rotation_table(num_rot):
    """cos/sin of the E-step angles ``j*pi/num_rot`` (emc.py:192), shape (R, 2)."""
    ang = np.arange(num_rot) * np.pi / num_rot
    return np.ascontiguousarray(np.stack([np.cos(ang), np.sin(ang)], axis=1))


def phaser_rotation_table(ang):
    """``(cos(-a), sin(-a))`` rows for the phaser's model->detector map,
    maxLP.py:309-311 and 255-258."""
    a = -np.asarray(ang, dtype='f8')
    return np.ascontiguousarray(np.stack([np.cos(a), np.sin(a)], axis=1))


def phaser_qvals(size):
    """q grids, radius, and the ``mask`` / ``rmask`` pixel sets, maxLP.py:79-95."""
    ind = (np.arange(size, dtype='f8') - size // 2) / size
    qx, qy = np.meshgrid(ind, ind, indexing='ij')
    qx, qy = qx.ravel(), qy.ravel()
    qrad = np.sqrt(qx * qx + qy * qy)
    qrad[qrad == 0] = 1.e-6
    mask = (qrad > 4 / size) & (qrad < 0.5)
    rmask = (qrad > 0.39) & (qrad < 0.41)
    return qx, qy, qrad, mask, rmask


def phaser_pixels(size):
    """Pixel lists of the two phaser passes and their histogram rows.

    Histogram rows cover ``mask | rmask`` in pixel order; ``mask_idx`` maps a
    pixel to its row (-1 elsewhere)."""
    _, _, _, mask, rmask = phaser_qvals(size)
    both = mask | rmask
    rows = np.flatnonzero(both).astype('i4')
    mask_idx = np.full(size * size, -1, dtype='i4')
    mask_idx[rows] = np.arange(rows.size, dtype='i4')
    ring = np.flatnonzero(rmask).astype('i4')
    main = np.flatnonzero(mask).astype('i4')
    return dict(mask=mask, rmask=rmask, mask_idx=mask_idx, n_rows=rows.size,
                ring=ring, ring_rows=mask_idx[ring], main=main, main_rows=mask_idx[main])
