"""FP64 NumPy oracle for the EMC E-step (rows a1-a10 of the hot path).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the checker for the
CUDA path, never part of it.

Conventions shared with the reference:
* pixels are row-major, ``t = x*size + y`` (kernels.cu:13, kernels.cu:52);
* states are the flattened ``meshgrid(sx, sy, dia, indexing='ij')``, so state
  ``s = (isx*nsy + isy)*nd + idia`` (emc.py:71-77);
* the likelihood row of (state s, rotation j) is ``s*num_rot + j``
  (emc.py:199).

Floating point is written operation by operation in the order of the
reference source, with no fused multiply-add (NumPy ufuncs never fuse), so
the CUDA kernels can reproduce integer-valued results (indices, argmax)
exactly by using ``__dmul_rn``/``__dadd_rn`` for the same expressions.
"""
import numpy as np

P_MIN = 1.e-6          # emc.py:20 (declared there, used here by the merge)
LOG_SENTINEL = -1000.  # kernels.cu:15,25,38


# --------------------------------------------------------------------------
# a1 / a2: sparse photon dataset (dset.py)
# --------------------------------------------------------------------------
def parse_photons(ones, multi, place_ones, place_multi, count_multi, num_pix,
                  need_scaling=False, bg=None):
    """Flat photon arrays + derived quantities, following dset.py:16-61.

    ``place_ones``/``place_multi``/``count_multi`` are the flattened vlen
    lists (np.hstack of the per-frame arrays, dset.py:34,43-44).  Returns a
    dict with the Dataset attribute names.  ``*_accum`` are int64 exclusive
    prefix sums (dset.py:32-33,41-42: ``roll(cumsum)`` with ``[0] = 0``).
    An empty dataset fails like the reference does (IndexError on ``[0]``).
    """
    ones = np.asarray(ones, dtype=np.int32)
    multi = np.asarray(multi, dtype=np.int32)
    place_ones = np.asarray(place_ones, dtype=np.int32)
    place_multi = np.asarray(place_multi, dtype=np.int32)
    count_multi = np.asarray(count_multi, dtype=np.int32)
    num_data = ones.shape[0]

    ones_accum = np.roll(np.cumsum(ones), 1)
    ones_accum[0] = 0
    multi_accum = np.roll(np.cumsum(multi), 1)
    multi_accum[0] = 0

    # dset.py:46-48
    mean_count = float((place_ones.shape[0] + count_multi.sum()) / num_data)
    counts = None
    if need_scaling:  # dset.py:50-53
        msum = np.array([count_multi[m_a:m_a + m].sum()
                         for m, m_a in zip(multi, multi_accum)], dtype=np.int64)
        counts = ones.astype(np.int64) + msum
    if bg is None:   # dset.py:56-60
        bg = np.zeros(num_pix)
    else:
        bg = np.asarray(bg, dtype=np.float64).ravel()
    return dict(num_data=num_data, num_pix=num_pix, ones=ones, multi=multi,
                ones_accum=ones_accum.astype(np.int64),
                multi_accum=multi_accum.astype(np.int64),
                place_ones=place_ones, place_multi=place_multi,
                count_multi=count_multi, mean_count=mean_count, counts=counts,
                bg=bg)


def get_powder(ds):
    """Mean photon count per pixel, dset.py:74-83 (``np.add.at`` then /N)."""
    powder = np.zeros(ds['num_pix'])
    np.add.at(powder, ds['place_ones'], 1)
    np.add.at(powder, ds['place_multi'], ds['count_multi'])
    powder /= ds['num_data']
    return powder


def get_scales(ds, need_scaling):
    """Per-frame scale factors, emc.py:129-132."""
    if need_scaling:
        return ds['counts'] / ds['mean_count']
    return np.ones(ds['num_data'], dtype='f8')


def frame_counts(ds, d):
    """Dense photon counts of frame d (dset.py:63-72 ``get_frame``)."""
    frame = np.zeros(ds['num_pix'], dtype='i4')
    o_a, m_a = ds['ones_accum'][d], ds['multi_accum'][d]
    np.add.at(frame, ds['place_ones'][o_a:o_a + ds['ones'][d]], 1)
    np.add.at(frame, ds['place_multi'][m_a:m_a + ds['multi'][d]],
              ds['count_multi'][m_a:m_a + ds['multi'][d]])
    return frame


def sparse_frames(ds, sel=None):
    """CSR (N x P) photon-count matrix, duplicates summed (maxLP.py:60-70).

    With ``sel`` (bool mask over pixels), columns outside ``sel`` are
    dropped and the remaining columns are renumbered in pixel order.
    """
    from scipy import sparse
    n, p = ds['num_data'], ds['num_pix']
    rows_o = np.repeat(np.arange(n), ds['ones'])
    rows_m = np.repeat(np.arange(n), ds['multi'])
    rows = np.concatenate([rows_o, rows_m])
    cols = np.concatenate([ds['place_ones'], ds['place_multi']]).astype(np.int64)
    vals = np.concatenate([np.ones(ds['place_ones'].shape[0]),
                           ds['count_multi'].astype(np.float64)])
    mat = sparse.csr_matrix((vals, (rows, cols)), shape=(n, p))
    mat.sum_duplicates()
    if sel is not None:
        mat = mat[:, np.where(sel)[0]]
    return mat.tocsr()


# --------------------------------------------------------------------------
# a3: states and masks (emc.py:67-98)
# --------------------------------------------------------------------------
def parse_triple(text):
    """``"lo hi n"`` config triple, emc.py:68-70."""
    return tuple(float(s) for s in text.split())


def generate_states(sx, sy, dia):
    """Flattened (shiftx, shifty, sphere_dia) grids, emc.py:71-78."""
    gx, gy, gd = np.meshgrid(np.linspace(sx[0], sx[1], int(sx[2])),
                             np.linspace(sy[0], sy[1], int(sy[2])),
                             np.linspace(dia[0], dia[1], int(dia[2])),
                             indexing='ij')
    num_states = np.array([sx[-1], sy[-1], dia[-1]]).astype('i4')
    return gx.ravel(), gy.ravel(), gd.ravel(), num_states


def detector_radius(size):
    """Integer-centred pixel radius, emc.py:81-84."""
    x_ind, y_ind = np.indices((size, size), dtype='f8')
    x_ind = x_ind.ravel() - size // 2
    y_ind = y_ind.ravel() - size // 2
    return x_ind, y_ind, np.sqrt(x_ind * x_ind + y_ind * y_ind)


def generate_masks(size):
    """``invmask`` and ``probmask`` (emc.py:89-98).  The likelihood uses the
    pixels with ``probmask < 1`` (kernels.cu:129,134)."""
    _, _, rad = detector_radius(size)
    invmask = np.zeros(size ** 2, dtype=bool)
    invmask[rad < 4] = True
    invmask[rad >= size // 2] = True
    probmask = np.zeros(size ** 2, dtype='i4')
    probmask[rad >= size // 2] = 2
    probmask[rad < size // 8] = 1
    probmask[rad < 4] = 2
    return invmask, probmask


# --------------------------------------------------------------------------
# a4: holographic slice (kernels.cu:44-82)
# --------------------------------------------------------------------------
def holo_slice(model, shiftx, shifty, diameter, rel_scale, scale, size, bg):
    """``slice_gen_holo`` with ``log_flag=0``: scale*|M + rel*ff*ramp|^2 + bg.

    kernels.cu:58-75.  ``|z|^2`` is evaluated as re*re + im*im.
    """
    model = np.asarray(model, dtype=np.complex128).ravel()
    x, y = np.indices((size, size), dtype='f8')
    x, y = x.ravel(), y.ravel()
    cen = np.floor(size / 2.)
    dx, dy = x - cen, y - cen
    phase = 2. * np.pi * (dx * shiftx + dy * shifty) / size
    s = np.sqrt(dx * dx + dy * dy) * np.pi * diameter / size
    s = np.where(s == 0., 1.e-5, s)
    sphere = rel_scale * (np.sin(s) - s * np.cos(s)) / (s * s * s)
    re = np.cos(phase) * sphere + model.real
    im = np.sin(phase) * sphere + model.imag
    view = re * re + im * im
    view = view * scale
    return view + bg


# --------------------------------------------------------------------------
# a6: rotated log slice (kernels.cu:6-42)
# --------------------------------------------------------------------------
def rotation_geometry(angle, size):
    """Bilinear source coordinates of ``slice_gen`` for one angle.

    kernels.cu:19-28: ``tx = (x-cen)*cos - (y-cen)*sin + cen``,
    ``ty = (x-cen)*sin + (y-cen)*cos + cen`` with integer ``cen = size/2``,
    ``ix = floor(tx)``; pixels whose 2x2 footprint leaves the detector are
    invalid.
    """
    x, y = np.indices((size, size))
    x, y = x.ravel(), y.ravel()
    cen = size // 2
    ac, as_ = np.cos(angle), np.sin(angle)
    xc = (x - cen).astype('f8')
    yc = (y - cen).astype('f8')
    tx = xc * ac - yc * as_ + cen
    ty = xc * as_ + yc * ac + cen
    ix = np.floor(tx).astype(np.int64)
    iy = np.floor(ty).astype(np.int64)
    valid = (ix >= 0) & (ix <= size - 2) & (iy >= 0) & (iy <= size - 2)
    fx, fy = tx - ix, ty - iy
    return ix, iy, fx, fy, valid


def rotate_slice(view, angle, scale, size, bg, log_flag):
    """``slice_gen`` (kernels.cu:6-42), vectorised over pixels."""
    view = np.asarray(view, dtype='f8').ravel()
    ix, iy, fx, fy, valid = rotation_geometry(angle, size)
    ixc = np.where(valid, ix, 0)
    iyc = np.where(valid, iy, 0)
    cx, cy = 1. - fx, 1. - fy
    out = (view[ixc * size + iyc] * cx * cy +
           view[(ixc + 1) * size + iyc] * fx * cy +
           view[ixc * size + (iyc + 1)] * cx * fy +
           view[(ixc + 1) * size + (iyc + 1)] * fx * fy)
    out = out * scale
    out = out + bg
    if log_flag:
        small = out < 1.e-20
        with np.errstate(divide='ignore', invalid='ignore'):
            out = np.where(small, LOG_SENTINEL, np.log(np.where(small, 1., out)))
        return np.where(valid, out, LOG_SENTINEL)
    return np.where(valid, out, 0.)


def rotation_angles(num_rot):
    """In-plane angles searched by the E-step: ``j*pi/num_rot`` (emc.py:192)."""
    return np.arange(num_rot) * np.pi / num_rot


# --------------------------------------------------------------------------
# a5 + a6 + a7: log-likelihood of every (state, rotation, frame)
# --------------------------------------------------------------------------
def msum_vscale(model, shiftx, shifty, sphere_dia, size, bg, probmask, powder):
    """Per-state masked slice sums and the global ``vscale``, emc.py:166-181.

    ``msums[i] = W_i[sel].sum()`` over the unrotated slice and
    ``vscale = powder[sel].sum() / sum_i W_i[sel].sum() * S0``.
    """
    sel = probmask < 1
    n_states = shiftx.shape[0]
    msums = np.empty(n_states)
    sum_views = np.zeros(size ** 2)
    for i in range(n_states):
        w = holo_slice(model, shiftx[i], shifty[i], sphere_dia[i], 1., 1., size, bg)
        msums[i] = w[sel].sum()
        sum_views += w
    vscale = powder[sel].sum() / sum_views[sel].sum() * n_states
    return msums, vscale


def log_slices_for_state(model, sx, sy, dia, size, bg, num_rot, sel):
    """Rotated log-slices of one (shift, diameter) state restricted to the
    likelihood pixels: array (num_rot, n_sel).  emc.py:186-193."""
    w = holo_slice(model, sx, sy, dia, 1., 1., size, bg)
    angles = rotation_angles(num_rot)
    out = np.empty((num_rot, int(sel.sum())))
    for j in range(num_rot):
        out[j] = rotate_slice(w, angles[j], 1., size, bg, 1)[sel]
    return out


def calc_prob(model, ds, shiftx, shifty, sphere_dia, size, num_rot, probmask,
              scales, states=None, frames=None):
    """Full likelihood matrix ``prob`` (S0*num_rot x N), emc.py:159-205 with
    calc_prob_all (kernels.cu:116-137):

    ``prob[s*R+j, d] = -msum_s*vscale*scale_d + sum_{p in frame d, probmask<1} K_d(p) L_{s,j}(p)``

    ``states``/``frames`` restrict the rows/columns computed (the full
    ``vscale`` is still computed over every state).
    """
    bg = ds['bg']
    powder = get_powder(ds)
    sel = probmask < 1
    msums, vscale = msum_vscale(model, shiftx, shifty, sphere_dia, size, bg,
                                probmask, powder)
    kmat = sparse_frames(ds, sel)
    if frames is not None:
        kmat = kmat[frames]
        scales = scales[frames]
    if states is None:
        states = range(shiftx.shape[0])
    states = list(states)
    prob = np.empty((len(states) * num_rot, kmat.shape[0]))
    for i, s in enumerate(states):
        lsl = log_slices_for_state(model, shiftx[s], shifty[s], sphere_dia[s],
                                   size, bg, num_rot, sel)
        init = -float(msums[s] * vscale)
        ll = np.asarray(kmat @ lsl.T).T          # (num_rot, N)
        prob[i * num_rot:(i + 1) * num_rot] = init * scales[None, :] + ll
    return prob, msums, vscale


def calc_prob_modes(models, ds, shiftx, shifty, sphere_dia, size, num_rot, probmask,
                    scales, frames=None):
    """Likelihood matrix for several models (``num_modes``, parsed at
    emc.py:59 and unused there; build-defined).  The (mode, state) pairs form
    the state list of emc.py:166-199: row ``(m*S0 + s)*num_rot + j`` holds
    model m in state s, and ``vscale`` is the one of emc.py:181 over all
    ``M*S0`` pairs, ``powder[sel].sum() / sum_pairs W[sel].sum() * M*S0``.
    With one model this is ``calc_prob``."""
    bg = ds['bg']
    powder = get_powder(ds)
    sel = probmask < 1
    n0 = shiftx.shape[0]
    msums, sums = [], []
    for model in models:
        ms, _ = msum_vscale(model, shiftx, shifty, sphere_dia, size, bg, probmask, powder)
        msums.append(ms)
        sums.append(ms.sum())
    msums = np.concatenate(msums)
    vscale = powder[sel].sum() / np.sum(sums) * (len(models) * n0)
    kmat = sparse_frames(ds, sel)
    if frames is not None:
        kmat = kmat[frames]
        scales = scales[frames]
    prob = np.empty((len(models) * n0 * num_rot, kmat.shape[0]))
    for m, model in enumerate(models):
        for s in range(n0):
            lsl = log_slices_for_state(model, shiftx[s], shifty[s], sphere_dia[s],
                                       size, bg, num_rot, sel)
            init = -float(msums[m * n0 + s] * vscale)
            r0 = (m * n0 + s) * num_rot
            prob[r0:r0 + num_rot] = init * scales[None, :] + np.asarray(kmat @ lsl.T).T
    return prob, msums, vscale


# --------------------------------------------------------------------------
# a8: most likely state per frame (emc.py:207-224)
# --------------------------------------------------------------------------
def get_rmax(prob):
    """Per-frame max and first-index argmax over states (emc.py:208-209;
    the MPI remap at emc.py:210 is the identity for one rank)."""
    return prob.max(0), prob.argmax(axis=0).astype('i4')


def unravel_rmax(rmax, shiftx, shifty, sphere_dia, num_states, num_rot):
    """Grid values of the chosen states, emc.py:218-224."""
    sx, sy, dia, ang = np.unravel_index(rmax, tuple(num_states) + (num_rot,))
    sx_vals = np.unique(shiftx)[sx]
    sy_vals = np.unique(shifty)[sy]
    dia_vals = np.unique(sphere_dia)[dia]
    ang_vals = ang * np.pi / num_rot
    return sx_vals, sy_vals, dia_vals, ang_vals


# --------------------------------------------------------------------------
# a9: per-frame posterior normalisation (build-defined, standard EMC)
# --------------------------------------------------------------------------
def posterior(prob):
    """``logZ_d = logsumexp_s prob[s,d]`` and ``P[s,d] = exp(prob - logZ)``.

    Not in the reference run path (it takes a hard argmax, emc.py:207-216);
    this is the standard EMC normalisation in FP64.
    """
    mx = prob.max(0)
    logz = mx + np.log(np.exp(prob - mx[None, :]).sum(0))
    return logz, np.exp(prob - logz[None, :])


# --------------------------------------------------------------------------
# a10: posterior-weighted merge (build-defined from merge_all + slice_merge)
# --------------------------------------------------------------------------
def slice_merge(view, angle, size, model, mweights):
    """Adjoint of ``slice_gen``: kernels.cu:84-114 (bilinear scatter of
    ``view`` into ``model`` and of the weights into ``mweights``)."""
    ix, iy, fx, fy, valid = rotation_geometry(angle, size)
    view = np.asarray(view, dtype='f8').ravel()
    cx, cy = 1. - fx, 1. - fy
    v = valid
    for (ox, oy, wgt) in ((0, 0, cx * cy), (1, 0, fx * cy), (0, 1, cx * fy), (1, 1, fx * fy)):
        idx = (ix[v] + ox) * size + (iy[v] + oy)
        np.add.at(model, idx, view[v] * wgt[v])
        np.add.at(mweights, idx, wgt[v])


def merge(prob_post, ds, scales, n_states0, num_rot, size, p_min=P_MIN):
    """Posterior-weighted merge into per-(shift, diameter) intensities.

    For state (s, j): data-space sum ``V_sj(p) = sum_d P[sj,d] K_d(p)``
    (merge_all, kernels.cu:139-152) over posteriors ``P >= p_min`` and
    weight ``w_sj = sum_d P[sj,d]*scale_d``; then the back-rotation
    (slice_merge, kernels.cu:84-114) accumulates
    ``num_s = sum_j R_j^T V_sj`` and ``den_s = sum_j w_sj R_j^T 1``.
    Returns ``intens = num/den`` (0 where den == 0), shape (S0, P), and
    ``num``, ``den``.
    """
    kmat = sparse_frames(ds)
    p = np.where(prob_post >= p_min, prob_post, 0.)
    vdata = np.asarray((kmat.T @ p.T).T)            # (S, P): sum_d P K_d
    wts = p @ scales                                 # (S,)
    num = np.zeros((n_states0, size * size))
    den = np.zeros((n_states0, size * size))
    angles = rotation_angles(num_rot)
    ones = np.ones(size * size)
    for s in range(n_states0):
        for j in range(num_rot):
            r = s * num_rot + j
            if wts[r] == 0.:
                continue
            dummy = np.zeros(size * size)
            slice_merge(vdata[r], angles[j], size, num[s], dummy)
            slice_merge(ones * wts[r], angles[j], size, den[s], dummy)
    intens = np.divide(num, den, out=np.zeros_like(num), where=den > 0)
    return intens, num, den
