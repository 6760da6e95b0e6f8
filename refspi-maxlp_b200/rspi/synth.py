"""Seeded synthetic holographic SPI data in the reference's photon layout.

The generative model (per frame d):

* sample: a real, positive 2-D density of ``n_blobs`` Gaussian blobs
  (sigma ~ U(1,3) px, amplitude ~ U(0.5,1), centres uniform in a disc of
  radius ``obj_radius`` px about ``size//2``), Fourier transformed with the
  ``fftshift(fftn(ifftshift(.)))`` convention (make_data.py:283);
* reference: a uniform sphere, ``rel * ff(pi*r*dia/size) * exp(2*pi*i*((x-c)*sx + (y-c)*sy)/size)``
  with ``ff(s) = (sin s - s cos s)/s^3`` exactly as slice_gen_holo builds it
  (kernels.cu:58-71); ``rel`` is set so that the mean |F_ref|^2 over the
  likelihood annulus equals the mean |F_sample|^2 there;
* per frame: diameter ~ U(dia_lo, dia_hi), shift ~ U(-shift_max, shift_max)^2,
  in-plane angle ~ U(0, 2 pi), fluence scale ~ lognormal(0, fluence_sigma);
* intensity ``|F_sample + F_ref|^2``, detector mask (r < 4 and r >= size//2
  set to 0, make_data.py:216-219), one global factor so the mean expected
  photon count is ``mean_count``, times the frame's scale, rotated with the
  bilinear ``slice_gen`` convention (kernels.cu:19-33), Poisson-sampled and
  stored as ``ones`` / ``multi`` lists (make_data.py:323-328).

Heterogeneous samples (``n_modes`` > 1): conformation 0 is the blob
density above; each further conformation displaces a fraction
``displace_frac`` of the blobs by ``displace`` px (uniform length, random
direction).  Each frame draws its conformation with ``mode_weights``.
Uneven loads (``count_lognormal = (median, sigma, lo, hi)``): each frame's
expected photon count is its own lognormal draw clipped to [lo, hi] instead
of the global normalisation times the fluence scale.  Background
(``bg_level``): that many expected photons on every detector pixel, added in
the detector frame after rotation and returned as ``bg`` (the photons
file's background model, dset.py:56-60); ``mean_count`` includes it.

Heavy per-frame work runs in torch on the requested device; the per-frame
parameters come from ``numpy.random.default_rng(seed)`` child streams.
"""
import numpy as np
import torch

CONFIGS = {
    # small plain-method case: 101x101, 1,000 frames, 500 photons/frame
    1: dict(size=101, n_blobs=20, obj_radius=12., num_data=1000, mean_count=500.,
            fluence_sigma=0.3, dia=(6., 8.), shift_max=3.,
            recon=dict(num_rot=180, shiftx='-3 3 7', shifty='-3 3 7',
                       sphere_dia='6 8 5', num_iter=10)),
    # production shape: 185x185, 20,000 frames, 2,000 photons/frame
    2: dict(size=185, n_blobs=40, obj_radius=20., num_data=20000, mean_count=2000.,
            fluence_sigma=0.5, dia=(6., 8.), shift_max=3.,
            recon=dict(num_rot=180, shiftx='-4 4 9', shifty='-4 4 9',
                       sphere_dia='6 8 5', num_iter=20)),
    # uneven load, heterogeneous sample: 185x185, 50,000 frames with
    # lognormal photon counts in [50, 50,000], 3 conformations (15% of blobs
    # displaced 2-4 px) with weights 0.5/0.3/0.2, reconstructed as 3 modes
    4: dict(size=185, n_blobs=40, obj_radius=20., num_data=50000, mean_count=None,
            fluence_sigma=0.5, dia=(6., 8.), shift_max=3., n_modes=3,
            mode_weights=(0.5, 0.3, 0.2), displace=(2., 4.), displace_frac=0.15,
            count_lognormal=(float(np.sqrt(50. * 50000.)), 1.15, 50., 50000.),
            recon=dict(num_rot=180, shiftx='-4 4 9', shifty='-4 4 9',
                       sphere_dia='6 8 5', num_iter=20, num_modes=3)),
    # dense high fluence: 255x255, 10,000 frames at 2e5 photons/frame stored
    # as dense uint16; a flat background of 2 photons per detector pixel
    # makes more than 80% of the pixels nonzero
    5: dict(size=255, n_blobs=40, obj_radius=20., num_data=10000, mean_count=2e5,
            fluence_sigma=0.3, dia=(6., 8.), shift_max=3., bg_level=2.0, dense=True,
            recon=dict(num_rot=360, shiftx='-5 5 11', shifty='-5 5 11',
                       sphere_dia='6 8 7', num_iter=10)),
}


def make_blobs(size, n_blobs, obj_radius, rng):
    """Blob centres, widths and amplitudes: (n_blobs, 4) = cx, cy, sigma, amp."""
    c = size // 2
    out = np.empty((n_blobs, 4))
    for b in range(n_blobs):
        r = obj_radius * np.sqrt(rng.random())
        phi = 2 * np.pi * rng.random()
        out[b] = (c + r * np.cos(phi), c + r * np.sin(phi), rng.uniform(1., 3.),
                  rng.uniform(0.5, 1.))
    return out


def render_blobs(size, blobs):
    x, y = np.indices((size, size), dtype='f8')
    obj = np.zeros((size, size))
    for cx, cy, sig, amp in blobs:
        obj += amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig ** 2))
    return obj


def make_object(size, n_blobs, obj_radius, rng):
    """Real positive density of Gaussian blobs centred on ``size//2``."""
    return render_blobs(size, make_blobs(size, n_blobs, obj_radius, rng))


def displaced_blobs(blobs, frac, dist, rng):
    """A conformation: ``frac`` of the blobs moved by U(dist) px."""
    out = blobs.copy()
    k = max(1, int(round(frac * len(blobs))))
    idx = rng.choice(len(blobs), size=k, replace=False)
    length = rng.uniform(dist[0], dist[1], k)
    phi = rng.uniform(0., 2 * np.pi, k)
    out[idx, 0] += length * np.cos(phi)
    out[idx, 1] += length * np.sin(phi)
    return out


def fourier(obj):
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(obj)))


def _sphere_ff(size, dia, device):
    """ff(pi*r*dia/size) per pixel (kernels.cu:66-69), dia: (B,) tensor."""
    x = torch.arange(size, dtype=torch.float64, device=device)
    cen = float(np.floor(size / 2.))
    dx = (x - cen)[:, None].expand(size, size).reshape(-1)
    dy = (x - cen)[None, :].expand(size, size).reshape(-1)
    r = torch.sqrt(dx * dx + dy * dy)
    s = r[None, :] * np.pi * dia[:, None] / size
    s = torch.where(s == 0, torch.full_like(s, 1e-5), s)
    return (torch.sin(s) - s * torch.cos(s)) / (s * s * s), dx, dy


def _rotate_bilinear(img, angle, size):
    """``slice_gen`` (no log): view[t] = bilinear(img)(R(angle)(t-c)+c), 0 outside."""
    b = img.shape[0]
    dev = img.device
    x = torch.arange(size, device=dev, dtype=torch.float64)
    cen = size // 2
    xc = (x - cen)[:, None].expand(size, size).reshape(-1)
    yc = (x - cen)[None, :].expand(size, size).reshape(-1)
    ac, as_ = torch.cos(angle)[:, None], torch.sin(angle)[:, None]
    tx = xc[None] * ac - yc[None] * as_ + cen
    ty = xc[None] * as_ + yc[None] * ac + cen
    ix, iy = torch.floor(tx), torch.floor(ty)
    valid = (ix >= 0) & (ix <= size - 2) & (iy >= 0) & (iy <= size - 2)
    fx, fy = tx - ix, ty - iy
    ix = torch.where(valid, ix, torch.zeros_like(ix)).long()
    iy = torch.where(valid, iy, torch.zeros_like(iy)).long()
    g = lambda a, c: torch.gather(img, 1, a * size + c)  # noqa: E731
    out = (g(ix, iy) * (1 - fx) * (1 - fy) + g(ix + 1, iy) * fx * (1 - fy) +
           g(ix, iy + 1) * (1 - fx) * fy + g(ix + 1, iy + 1) * fx * fy)
    return torch.where(valid, out, torch.zeros_like(out)).reshape(b, -1)


def generate(size, num_data, mean_count, n_blobs=20, obj_radius=12.,
             fluence_sigma=0.3, dia=(6., 8.), shift_max=3., seed=0,
             device='cpu', chunk=256, dense=False, n_modes=1, mode_weights=None,
             displace=(2., 4.), displace_frac=0.15, count_lognormal=None, bg_level=0.,
             frame_seed=None):
    """Generate one dataset; returns a dict in the photons-file layout.

    Keys: ``num_pix``, ``ones``, ``multi`` (int32, N), ``place_ones``,
    ``place_multi``, ``count_multi`` (flat int32; per-frame lengths are
    ``ones``/``multi``), truth ``true_angles``, ``true_shifts``,
    ``true_diameters``, ``scale``, ``solution``, and ``fsample``/``rel_scale``.
    With ``n_modes`` > 1, ``solution``/``fsample`` hold one row per
    conformation and ``true_modes`` each frame's.  With ``dense=True`` a
    dense uint16 ``frames`` (N, size^2) is added.  ``frame_seed`` draws
    other frames (parameters and photons) of the same object.
    """
    ss = np.random.SeedSequence(seed)
    r_obj, r_par, r_poi = [np.random.default_rng(s) for s in ss.spawn(3)]
    if frame_seed is not None:
        # the same object, other frames (parameters and photon draws)
        r_par, r_poi = [np.random.default_rng(s)
                        for s in np.random.SeedSequence([seed, frame_seed]).spawn(2)]
    blobs = [make_blobs(size, n_blobs, obj_radius, r_obj)]
    for _ in range(1, n_modes):
        blobs.append(displaced_blobs(blobs[0], displace_frac, displace, r_obj))
    objs = [render_blobs(size, b) for b in blobs]
    fss = [fourier(o).ravel() for o in objs]

    diam = r_par.uniform(dia[0], dia[1], num_data)
    shifts = r_par.uniform(-shift_max, shift_max, (num_data, 2))
    angles = r_par.uniform(0., 2 * np.pi, num_data)
    scale = r_par.lognormal(0., fluence_sigma, num_data)
    modes = np.zeros(num_data, dtype='i4')
    if n_modes > 1:
        wts = np.full(n_modes, 1. / n_modes) if mode_weights is None else np.asarray(mode_weights)
        modes = r_par.choice(n_modes, size=num_data, p=wts / wts.sum()).astype('i4')
    target = None
    if count_lognormal is not None:
        med, sig, lo_c, hi_c = count_lognormal
        target = np.clip(r_par.lognormal(np.log(med), sig, num_data), lo_c, hi_c)
        scale = target / target.mean()

    dev = torch.device(device)
    fs_all = torch.from_numpy(np.stack(fss)).to(dev)
    fs_t = fs_all[0]
    modes_t = torch.from_numpy(modes.astype(np.int64)).to(dev)
    x = torch.arange(size, dtype=torch.float64, device=dev)
    cen = size // 2
    pr = torch.sqrt(((x - cen)[:, None] ** 2 + (x - cen)[None, :] ** 2)).reshape(-1)
    detmask = ((pr >= 4) & (pr < cen)).double()
    llmask = (pr >= max(size // 8, 4)) & (pr < size // 2)

    ff0, dx, dy = _sphere_ff(size, torch.tensor([0.5 * (dia[0] + dia[1])], device=dev,
                                                dtype=torch.float64), dev)
    rel = float(torch.sqrt((fs_t.abs() ** 2)[llmask].mean() / (ff0[0] ** 2)[llmask].mean()))

    def intens(lo, hi):
        d = torch.from_numpy(diam[lo:hi]).to(dev)
        sh = torch.from_numpy(shifts[lo:hi]).to(dev)
        ff, _, _ = _sphere_ff(size, d, dev)
        ph = 2. * np.pi * (dx[None] * sh[:, :1] + dy[None] * sh[:, 1:]) / size
        fsm = fs_all[modes_t[lo:hi]]
        re = torch.cos(ph) * ff * rel + fsm.real
        im = torch.sin(ph) * ff * rel + fsm.imag
        return (re * re + im * im) * detmask[None]

    bgmap = bg_level * detmask
    if target is None:
        tot = 0.
        for lo in range(0, num_data, chunk):
            hi = min(num_data, lo + chunk)
            w = intens(lo, hi).sum(1).cpu().numpy()
            tot += float((w * scale[lo:hi]).sum())
        signal = mean_count - float(bgmap.sum())
        if signal <= 0:
            raise ValueError('the background alone exceeds mean_count')
        gfac = signal * num_data / tot

    gen = torch.Generator(device=dev)
    gen.manual_seed(int(r_poi.integers(0, 2 ** 62)))
    ones, multi = np.zeros(num_data, 'i4'), np.zeros(num_data, 'i4')
    po, pm, cm = [], [], []
    frames = np.zeros((num_data, size * size), dtype=np.uint16) if dense else None
    for lo in range(0, num_data, chunk):
        hi = min(num_data, lo + chunk)
        w = intens(lo, hi)
        if target is None:
            w = w * (gfac * torch.from_numpy(scale[lo:hi]).to(dev))[:, None]
        else:   # this frame's own expected count
            w = w * (torch.from_numpy(target[lo:hi]).to(dev) / w.sum(1))[:, None]
        rot = _rotate_bilinear(w, torch.from_numpy(angles[lo:hi]).to(dev), size)
        if bg_level:
            rot = rot + bgmap[None]
        cnt = torch.poisson(rot, generator=gen).to(torch.int32)
        if dense:
            frames[lo:hi] = cnt.clamp(max=65535).cpu().numpy().astype(np.uint16)
        # row-major nonzeros: frame by frame, pixels ascending (np.flatnonzero order)
        nz = torch.nonzero(cnt)
        val = cnt[nz[:, 0], nz[:, 1]]
        one = val == 1
        ones[lo:hi] = torch.bincount(nz[one, 0], minlength=hi - lo).cpu().numpy()
        multi[lo:hi] = torch.bincount(nz[~one, 0], minlength=hi - lo).cpu().numpy()
        po.append(nz[one, 1].to(torch.int32).cpu().numpy())
        pm.append(nz[~one, 1].to(torch.int32).cpu().numpy())
        cm.append(val[~one].cpu().numpy().astype('i4'))
    cat = lambda a: np.concatenate(a) if a else np.zeros(0, 'i4')  # noqa: E731
    out = dict(num_pix=np.array([size * size]), ones=ones, multi=multi,
               place_ones=cat(po), place_multi=cat(pm), count_multi=cat(cm),
               true_angles=angles, true_shifts=shifts, true_diameters=diam,
               scale=scale, solution=objs[0] if n_modes == 1 else np.stack(objs),
               fsample=fss[0] if n_modes == 1 else np.stack(fss), rel_scale=np.array(rel))
    if n_modes > 1:
        out['true_modes'] = modes
    if bg_level:
        out['bg'] = bgmap.cpu().numpy()
    if dense:
        out['frames'] = frames
    return out


def generate_config(cfg, device='cpu', num_data=None, seed=None):
    """Dataset of a named configuration (seeded by ``20260000 + cfg``)."""
    c = CONFIGS[cfg]
    return generate(c['size'], c['num_data'] if num_data is None else num_data,
                    c['mean_count'], c['n_blobs'], c['obj_radius'], c['fluence_sigma'],
                    c['dia'], c['shift_max'], seed=20260000 + cfg if seed is None else seed,
                    device=device, **config_extras(cfg))


def config_extras(cfg):
    """Keyword arguments of ``generate`` beyond the common ones."""
    c = CONFIGS[cfg]
    return {k: c[k] for k in ('n_modes', 'mode_weights', 'displace', 'displace_frac',
                              'count_lognormal', 'bg_level', 'dense') if k in c}


def initial_model(size, seed):
    """Random complex start model U[0,1) + iU[0,1) (emc.py:241-242), seeded."""
    rng = np.random.default_rng(seed)
    return rng.random(size ** 2) + 1j * rng.random(size ** 2)
