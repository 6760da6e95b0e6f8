"""Replay of the reference's GPU code path on one B200 (test and baseline
infrastructure only; see ``oracle/__init__.py``).

The reference runs with CuPy, which is not installed here.  This module
runs the same loops with the reference's own kernels (``kernels.cu``,
compiled by ``oracle/ref_gpu/build.py``) and torch tensors in place of
CuPy arrays:

* ``estep``: ``EMC._calculate_prob`` (emc.py:159-205): per (shift, diameter)
  state ``slice_gen_holo`` on one of four streams, the masked sums and
  vscale (emc.py:174-181), then per rotation ``slice_gen`` (log) and
  ``calc_prob_all`` with the reference's grids and blocks.
* ``run_pixel_pattern`` / ``run_phaser_pixels``: ``MaxLPhaser``'s pattern
  search (maxLP.py:154-228, 304-340): the reference's ``get_f_dt`` kernel
  for the frames x candidates amplitudes, then the CuPy element-wise and
  reduction steps of ``get_logq_pixel`` / ``get_rescale_pixel`` as the same
  torch operations.  The photons of a pixel (``get_photons_pixel``,
  maxLP.py:245-253) are looked up in the CSR photon matrix with one sorted
  search (cupyx fancy indexing is not available); this lookup is once per
  pixel and does not change the per-iteration work.

The timing helpers measure a bounded sample of states / pixels on the GPU
with CUDA events and extrapolate linearly to a whole iteration.
"""
import ctypes
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(HERE), '_ref', 'libref_kernels_gpu.so')

_P, _L, _I, _U, _D = (ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_uint,
                      ctypes.c_double)
_lib = None


def load():
    """The reference kernels for the GPU; raises if they were not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError('%s is not built (oracle/ref_gpu/build.py)' % LIB)
        lib = ctypes.CDLL(LIB)
        lib.ref_gpu_slice_gen.argtypes = [_U, _U, _U, _U, _P, _D, _D, _L, _P, _L, _P, _P]
        lib.ref_gpu_slice_gen_holo.argtypes = [_U, _U, _U, _U, _P, _D, _D, _D, _D, _D, _L, _P,
                                               _L, _P, _P]
        lib.ref_gpu_calc_prob_all.argtypes = [_U, _U, _P, _P, _L, _P, _P, _P, _P, _P, _P, _P,
                                              _D, _P, _P, _P]
        lib.ref_gpu_get_f_dt.argtypes = [_U, _U, _P, _P, _L, _L, _P, _P]
        for f in (lib.ref_gpu_slice_gen, lib.ref_gpu_slice_gen_holo, lib.ref_gpu_calc_prob_all,
                  lib.ref_gpu_get_f_dt):
            f.restype = _I
        _lib = lib
    return _lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _ok(code, what):
    if code != 0:
        raise RuntimeError('%s: CUDA error %d' % (what, code))


class RefData:
    """The reference's device arrays (dset.py:23-60) as torch tensors."""

    def __init__(self, ones, multi, place_ones, place_multi, count_multi, size, bg, scales,
                 probmask, device):
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to(device, dt)  # noqa: E731
        self.size = int(size)
        self.n = len(ones)
        self.ones, self.multi = t(ones, torch.int32), t(multi, torch.int32)
        self.place_ones = t(place_ones, torch.int32)
        self.place_multi = t(place_multi, torch.int32)
        self.count_multi = t(count_multi, torch.int32)
        oa = np.concatenate([[0], np.cumsum(ones)[:-1]]).astype(np.int64)
        ma = np.concatenate([[0], np.cumsum(multi)[:-1]]).astype(np.int64)
        self.ones_accum, self.multi_accum = t(oa, torch.int64), t(ma, torch.int64)
        self.bg = t(bg, torch.float64)
        self.scales = t(scales, torch.float64)
        self.probmask = t(probmask.astype('i4'), torch.int32)
        npix = self.size ** 2
        powder = np.zeros(npix)
        np.add.at(powder, place_ones, 1.)
        np.add.at(powder, place_multi, count_multi)
        self.powder = t(powder / self.n, torch.float64)
        self.device = device
        # CSR photon matrix (frames x pixels), keys d * P + pixel ascending
        rows = np.repeat(np.arange(self.n), np.asarray(ones) + np.asarray(multi))
        cols = np.concatenate([np.concatenate([a, b]) for a, b in zip(
            np.split(place_ones, np.cumsum(ones)[:-1]), np.split(place_multi, np.cumsum(multi)[:-1]))]) \
            if self.n else np.zeros(0, np.int64)
        vals = np.concatenate([np.concatenate([np.ones(len(a)), b]) for a, b in zip(
            np.split(place_ones, np.cumsum(ones)[:-1]),
            np.split(np.asarray(count_multi, dtype='f8'), np.cumsum(multi)[:-1]))])
        keys = rows.astype(np.int64) * npix + cols.astype(np.int64)
        order = np.argsort(keys, kind='stable')
        self.csr_keys = t(keys[order], torch.int64)
        self.csr_vals = t(vals[order], torch.float64)


def estep(lib, data, model, shiftx, shifty, sphere_dia, num_rot, states=None, n_streams=4,
          prob=None):
    """``_calculate_prob`` of emc.py:159-205 with the reference's kernels.
    ``states`` restricts the likelihood rows computed (vscale is over all
    states, as the reference computes it).  Returns the (rows x frames)
    FP64 matrix of the states computed."""
    size, n, dev = data.size, data.n, data.device
    npix = size * size
    bm = (size + 31) // 32
    bd = (n + 31) // 32
    streams = [torch.cuda.Stream(dev) for _ in range(n_streams)]
    views = torch.empty((n_streams, npix), dtype=torch.float64, device=dev)
    rot_views = torch.empty_like(views)
    sel = data.probmask < 1
    n0 = len(shiftx)
    msums = torch.empty(n0, dtype=torch.float64, device=dev)
    sum_views = torch.zeros_like(views)
    cur = torch.cuda.current_stream(dev)
    for sst in streams:
        sst.wait_stream(cur)
    for i in range(n0):
        st = streams[i % n_streams]
        with torch.cuda.stream(st):
            _ok(lib.ref_gpu_slice_gen_holo(bm, bm, 32, 32, _p(model), float(shiftx[i]),
                                           float(shifty[i]), float(sphere_dia[i]), 1., 1., size,
                                           _p(data.bg), 0, _p(views[i % n_streams]),
                                           ctypes.c_void_p(st.cuda_stream)), 'slice_gen_holo')
            msums[i] = views[i % n_streams][sel].sum()
            sum_views[i % n_streams] += views[i % n_streams]
    for sst in streams:
        cur.wait_stream(sst)
    vscale = data.powder[sel].sum() / sum_views.sum(0)[sel].sum() * n0
    states = list(range(n0)) if states is None else list(states)
    if prob is None:
        prob = torch.empty((len(states) * num_rot, n), dtype=torch.float64, device=dev)
    for sst in streams:
        sst.wait_stream(cur)
    for k, i in enumerate(states):
        st = streams[k % n_streams]
        v, rv = views[k % n_streams], rot_views[k % n_streams]
        with torch.cuda.stream(st):
            sp = ctypes.c_void_p(st.cuda_stream)
            _ok(lib.ref_gpu_slice_gen_holo(bm, bm, 32, 32, _p(model), float(shiftx[i]),
                                           float(shifty[i]), float(sphere_dia[i]), 1., 1., size,
                                           _p(data.bg), 0, _p(v), sp), 'slice_gen_holo')
            init = -float(msums[i] * vscale)    # the reference reads msums[i] on the host
            for j in range(num_rot):
                _ok(lib.ref_gpu_slice_gen(bm, bm, 32, 32, _p(v), j * np.pi / num_rot, 1., size,
                                          _p(data.bg), 1, _p(rv), sp), 'slice_gen')
                _ok(lib.ref_gpu_calc_prob_all(
                    bd, 32, _p(rv), _p(data.probmask), n, _p(data.ones), _p(data.multi),
                    _p(data.ones_accum), _p(data.multi_accum), _p(data.place_ones),
                    _p(data.place_multi), _p(data.count_multi), init, _p(data.scales),
                    _p(prob[k * num_rot + j]), sp), 'calc_prob_all')
    for sst in streams:
        cur.wait_stream(sst)
    return prob


# ---------------------------------------------------------------------------
# MaxLP (maxLP.py:154-228, 304-340)
# ---------------------------------------------------------------------------
def pattern(device):
    ind = torch.arange(-8, 8.5, 0.5, dtype=torch.float64, device=device)
    x, y = torch.meshgrid(ind, ind, indexing='ij')
    return torch.complex(x, y).reshape(-1)


def pixel_constants(data, t, ang, shifts, diams):
    """k_d and fref_d of model pixel t (maxLP.py:107-114, 238-253)."""
    size, dev = data.size, data.device
    c0 = size // 2
    qx = (t // size - c0) / size
    qy = (t % size - c0) / size
    qrad = max(np.sqrt(qx * qx + qy * qy), 1e-6)
    c, s = torch.cos(-ang), torch.sin(-ang)
    x = torch.round((c * qx - s * qy) * size + c0).to(torch.int64)   # rint, half to even
    y = torch.round((s * qx + c * qy) * size + c0).to(torch.int64)
    tv = x * size + y
    keys = torch.arange(data.n, device=dev, dtype=torch.int64) * size * size + tv
    pos = torch.searchsorted(data.csr_keys, keys).clamp(max=max(0, data.csr_keys.numel() - 1))
    hit = data.csr_keys[pos] == keys if data.csr_keys.numel() else torch.zeros_like(keys, dtype=torch.bool)
    k_d = torch.where(hit, data.csr_vals[pos], torch.zeros((), dtype=torch.float64, device=dev))
    sval = np.pi * qrad * diams
    fref = (torch.sin(sval) - sval * torch.cos(sval)) / sval ** 3
    ramp = torch.exp(1j * 2 * np.pi * (qx * shifts[:, 0] + qy * shifts[:, 1]))
    return k_d, fref * ramp


def _f_dt(lib, cand, fref_d):
    n, nc = fref_d.numel(), cand.numel()
    f_dt = torch.empty((n, nc), dtype=torch.complex128, device=fref_d.device)
    _ok(lib.ref_gpu_get_f_dt((n + 31) // 32, 32, _p(cand), _p(fref_d), n, nc, _p(f_dt),
                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
        'get_f_dt')
    return f_dt


def rescale_pixel(lib, cand, k_d, fref_d):
    f_dt = _f_dt(lib, cand, fref_d)
    return k_d.mean() / (f_dt.abs() ** 2).mean(0)


def logq_pixel(lib, cand, k_d, fref_d, rescale=None):
    if rescale is None:
        rescale = rescale_pixel(lib, cand, k_d, fref_d)
    f_dt = _f_dt(lib, cand, fref_d)
    w_dt = rescale * f_dt.abs() ** 2
    return (k_d[:, None] * torch.log(w_dt)).mean(0) - w_dt.mean(0)


def run_pixel_pattern(lib, f_t, k_d, fref_d, pat, rescale=None, num_iter=10):
    f_t = complex(f_t)
    step = abs(f_t) / 4.
    centre = pat.numel() // 2
    for _ in range(num_iter):
        cand = (f_t + pat * step).contiguous()
        vals = logq_pixel(lib, cand, k_d, fref_d, rescale)
        imax = int(vals.argmax())
        f_new = f_t + complex(pat[imax]) * step
        step_new = step / (pat.numel() ** 0.5 / 5) if imax == centre else step
        if step_new / abs(f_new) < 1.e-3:
            break
        f_t, step = f_new, step_new
    return f_t


def time_iteration(lib, data, model, shiftx, shifty, sphere_dia, num_rot, n_states=4,
                   n_ring=8, n_main=16, seed=0):
    """Seconds per EMC iteration of the reference path on this GPU, from a
    bounded sample, extrapolated linearly: the vscale pass over every state
    plus ``n_states`` states x all rotations (E-step), and ``n_ring`` ring and
    ``n_main`` main-pass pixels of the phaser over all frames (M-step, with
    frames spread over the states and rotations at random)."""
    import time
    dev = data.device
    n0 = len(shiftx)

    def wall(f):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        f()
        torch.cuda.synchronize(dev)
        return time.perf_counter() - t0

    estep(lib, data, model, shiftx, shifty, sphere_dia, num_rot, states=[0])   # warm-up
    t_vs = wall(lambda: estep(lib, data, model, shiftx, shifty, sphere_dia, num_rot, states=[]))
    picks = np.linspace(0, n0 - 1, n_states).astype(int)
    prob = torch.empty((n_states * num_rot, data.n), dtype=torch.float64, device=dev)
    t_st = wall(lambda: estep(lib, data, model, shiftx, shifty, sphere_dia, num_rot,
                              states=picks, prob=prob)) - t_vs
    e_s = t_vs + max(t_st, 0.) / n_states * n0

    rng = np.random.default_rng(seed)
    st = rng.integers(0, n0, data.n)
    ang = torch.as_tensor(rng.integers(0, num_rot, data.n) * np.pi / num_rot).to(dev)
    shifts = torch.as_tensor(np.stack([np.asarray(shiftx)[st], np.asarray(shifty)[st]], 1)).to(dev)
    diams = torch.as_tensor(np.asarray(sphere_dia)[st]).to(dev)
    size = data.size
    q = (np.arange(size) - size // 2) / size
    qrad = np.sqrt(q[:, None] ** 2 + q[None, :] ** 2).ravel()
    qrad[qrad == 0] = 1e-6
    mask = (qrad > 4 / size) & (qrad < 0.5)
    rmask = (qrad > 0.39) & (qrad < 0.41)
    ring, main = np.flatnonzero(rmask), np.flatnonzero(mask)
    pat = pattern(dev)
    mflat = torch.as_tensor(np.asarray(model.cpu())).reshape(-1)

    def ring_pixel(t):
        k_d, fr = pixel_constants(data, int(t), ang, shifts, diams)
        f = run_pixel_pattern(lib, mflat[t].item(), k_d, fr, pat, None, 10)
        k_d, fr = pixel_constants(data, int(t), ang, shifts, diams)   # maxLP.py:326
        rescale_pixel(lib, torch.tensor([f], dtype=torch.complex128, device=dev), k_d, fr)

    def main_pixel(t):
        k_d, fr = pixel_constants(data, int(t), ang, shifts, diams)
        run_pixel_pattern(lib, mflat[t].item(), k_d, fr, pat, 1.0, 10)

    rs = ring[np.linspace(0, ring.size - 1, n_ring).astype(int)] if ring.size else []
    ms = main[np.linspace(0, main.size - 1, n_main).astype(int)]
    ring_pixel(rs[0]) if len(rs) else main_pixel(ms[0])   # warm-up
    t_ring = wall(lambda: [ring_pixel(t) for t in rs]) / max(1, len(rs))
    t_main = wall(lambda: [main_pixel(t) for t in ms]) / max(1, len(ms))
    m_s = t_ring * ring.size + t_main * main.size
    return dict(s_per_iteration=e_s + m_s, estep_s=e_s, mstep_s=m_s, vscale_pass_s=t_vs,
                s_per_state=max(t_st, 0.) / n_states, s_per_ring_pixel=t_ring,
                s_per_main_pixel=t_main,
                sample=('reference kernels.cu on this GPU: vscale pass over %d states + %d '
                        'states x %d rotations (E-step); %d ring + %d main-pass phaser pixels '
                        'over %d frames (M-step); linear extrapolation to %d states, %d ring '
                        'and %d main pixels' % (n0, n_states, num_rot, len(rs), len(ms),
                                                data.n, n0, ring.size, main.size)))
