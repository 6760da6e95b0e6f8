"""Device-resident data and the per-iteration pipelines over librspi.

``DevicePhotons``  photon lists on the GPU plus their derived arrays (a1, a2)
                   and the packed likelihood entry lists.
``EStep``          holographic slices -> vscale -> rotated log-slices ->
                   log-likelihood -> per-frame max/argmax/log-sum-exp (a4-a9).
``MStep``          photon histograms -> ring pass -> global rescale -> main
                   pass of the MaxLP pattern search (a11-a14).

Every call launches on torch's current CUDA stream and never synchronises
except where a host value is explicitly requested (``*_host`` helpers and
``check_errors``), so an iteration can be captured in a CUDA graph.
"""
import ctypes

import numpy as np
import torch

from . import geometry
from .lib import call, check, load

_f64 = torch.float64
_i32 = torch.int32
_i64 = torch.int64


def ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def cur_stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(device):
    if device is None:
        device = torch.device('cuda', torch.cuda.current_device())
    device = torch.device(device)
    if device.type != 'cuda':
        raise RuntimeError('the RefSPI-MaxLP kernels run on CUDA devices only')
    return device


class ErrorWord:
    """Device int32 that kernels set to the first RSPI_ERR_* they hit."""

    def __init__(self, device):
        self.t = torch.zeros(1, dtype=_i32, device=device)

    def check(self, what):
        code = int(self.t.item())
        if code != 0:
            self.t.zero_()
            check(code, what)


class DevicePhotons:
    """Sparse photons on the device (dset.py layout) and derived arrays."""

    def __init__(self, ones, multi, place_ones, place_multi, count_multi, num_pix,
                 need_scaling=False, device=None):
        self.lib = load()
        self.device = _dev(device)
        ones = np.ascontiguousarray(ones, dtype='i4')
        multi = np.ascontiguousarray(multi, dtype='i4')
        place_ones = np.ascontiguousarray(place_ones, dtype='i4')
        place_multi = np.ascontiguousarray(place_multi, dtype='i4')
        count_multi = np.ascontiguousarray(count_multi, dtype='i4')
        n = ones.shape[0]
        if n == 0:
            raise IndexError('index 0 is out of bounds for axis 0 with size 0')
        if multi.shape[0] != n:
            raise ValueError('ones and multi have different lengths')
        if ones.min() < 0 or multi.min() < 0:
            raise ValueError('negative photon count in ones/multi')
        if int(ones.sum(dtype=np.int64)) != place_ones.size:
            raise ValueError('sum(ones) != len(place_ones)')
        if int(multi.sum(dtype=np.int64)) != place_multi.size or place_multi.size != count_multi.size:
            raise ValueError('sum(multi), len(place_multi) and len(count_multi) disagree')
        for name, arr in (('place_ones', place_ones), ('place_multi', place_multi)):
            if arr.size and (arr.min() < 0 or arr.max() >= num_pix):
                raise ValueError('%s holds pixel indices outside [0, %d)' % (name, num_pix))
        self.num_data, self.num_pix = n, int(num_pix)
        self.need_scaling = bool(need_scaling)
        up = lambda a: torch.from_numpy(a).to(self.device)  # noqa: E731
        self.ones, self.multi = up(ones), up(multi)
        self.place_ones, self.place_multi, self.count_multi = up(place_ones), up(place_multi), up(count_multi)
        dev = self.device
        self.err = ErrorWord(dev)
        self.ones_accum = torch.empty(n, dtype=_i64, device=dev)
        self.multi_accum = torch.empty(n, dtype=_i64, device=dev)
        self.counts = torch.empty(n, dtype=_i64, device=dev)
        self.totals = torch.empty(3, dtype=_i64, device=dev)
        self.mean_count_t = torch.empty(1, dtype=_f64, device=dev)
        self.scales = torch.empty(n, dtype=_f64, device=dev)
        self.powder = torch.empty(self.num_pix, dtype=_f64, device=dev)
        s = cur_stream()
        call('rspi_photon_offsets', ptr(self.ones), ptr(self.multi), ptr(self.count_multi), n, ptr(self.ones_accum),
            ptr(self.multi_accum), ptr(self.counts), ptr(self.totals), ptr(self.mean_count_t),
            ptr(self.scales), int(self.need_scaling), ptr(self.err.t), s)
        call('rspi_powder', ptr(self.place_ones), place_ones.size, ptr(self.place_multi), ptr(self.count_multi),
            place_multi.size, self.num_pix, n, ptr(self.powder), ptr(self.err.t), s)
        self.err.check('photon set-up')
        self.mean_count = float(self.mean_count_t.item())
        self._ll = None

    def ll_entries(self, pix2sel, p_pad):
        """Packed likelihood entries for the given sel map (built once)."""
        key = (int(p_pad), pix2sel.data_ptr())
        if self._ll is not None and self._ll['key'] == key:
            return self._ll
        n, dev, s = self.num_data, self.device, cur_stream()
        frame_rows = torch.empty(n, dtype=_i32, device=dev)
        frame_sel = torch.empty(n, dtype=_i64, device=dev)
        call('rspi_ll_entry_rows', ptr(self.ones), ptr(self.multi), ptr(self.ones_accum), ptr(self.multi_accum),
            ptr(self.place_ones), ptr(self.place_multi), ptr(self.count_multi), ptr(pix2sel),
            self.num_pix, n, ptr(frame_rows), ptr(frame_sel), ptr(self.err.t), s)
        row_off = torch.empty(n + 1, dtype=_i64, device=dev)
        call('rspi_scan_rows', ptr(frame_rows), n, ptr(row_off), s)
        self.err.check('likelihood entry rows')
        total = int(row_off[-1].item())
        entries = torch.empty(max(1, total) * 32, dtype=_i32, device=dev)
        call('rspi_ll_entry_fill', ptr(self.ones), ptr(self.multi), ptr(self.ones_accum), ptr(self.multi_accum),
            ptr(self.place_ones), ptr(self.place_multi), ptr(self.count_multi), ptr(pix2sel),
            self.num_pix, n, ptr(row_off), ptr(entries), ptr(self.err.t), s)
        order = torch.argsort(frame_rows, descending=True, stable=True).to(_i32)
        self.err.check('likelihood entry fill')
        self._ll = dict(key=key, frame_rows=frame_rows, frame_sel_photons=frame_sel,
                        row_off=row_off, entries=entries, order=order, total_rows=total)
        return self._ll


class EStep:
    """Likelihood of every frame in every (shift, diameter, rotation) state."""

    def __init__(self, photons, size, num_rot, shiftx, shifty, sphere_dia, probmask, bg,
                 slice_dtype='f64', prob_dtype='f64', states_per_tile=None, warps=32,
                 n_ctas=0, slice_budget_bytes=8 << 30):
        self.lib = load()
        self.ph = photons
        self.device = dev = photons.device
        self.size, self.num_rot = int(size), int(num_rot)
        self.n_states0 = int(np.asarray(shiftx).size)
        self.n_rows = self.n_states0 * self.num_rot
        sel, pix2sel, p_pad = geometry.sel_pixels(probmask)
        self.n_sel, self.p_pad = sel.size, p_pad
        t = lambda a, dt=_f64: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        self.sel_pix, self.pix2sel = t(sel, _i32), t(pix2sel, _i32)
        self.shiftx, self.shifty, self.sphere_dia = t(shiftx), t(shifty), t(sphere_dia)
        self.rot_cs = t(geometry.emc_rotation_table(self.num_rot))
        self.bg = t(np.asarray(bg, dtype='f8').ravel())
        self.slice_code = {'f32': 0, 'f64': 1}[slice_dtype]
        self.prob_code = {'f32': 0, 'f64': 1}[prob_dtype]
        self.slice_torch = torch.float32 if self.slice_code == 0 else _f64
        self.prob_torch = torch.float32 if self.prob_code == 0 else _f64
        tmax = self.lib.rspi_loglike_max_tile(self.p_pad, self.slice_code)
        if tmax == 0:
            raise ValueError('a %d-pixel likelihood slice does not fit in shared memory' % self.n_sel)
        self.tile = int(states_per_tile or tmax)
        if self.tile > tmax:
            raise ValueError('states_per_tile %d exceeds the shared-memory limit %d' % (self.tile, tmax))
        self.warps, self.n_ctas = int(warps), int(n_ctas)
        self.ll = photons.ll_entries(self.pix2sel, self.p_pad)
        esz = 4 if self.slice_code == 0 else 8
        rows = max(self.tile, (slice_budget_bytes // (self.p_pad * esz)) // self.tile * self.tile)
        self.chunk_rows = int(min(self.n_rows, rows))
        self.holo = torch.empty((self.n_states0, self.size ** 2), dtype=_f64, device=dev)
        self.msum = torch.empty(self.n_states0, dtype=_f64, device=dev)
        self.vscale = torch.empty(1, dtype=_f64, device=dev)
        self.init = torch.empty(self.n_states0, dtype=_f64, device=dev)
        self.lsl = torch.empty((self.chunk_rows, self.p_pad), dtype=self.slice_torch, device=dev)
        self.prob = torch.empty((self.n_rows, photons.num_data), dtype=self.prob_torch, device=dev)
        self.maxll = torch.empty(photons.num_data, dtype=_f64, device=dev)
        self.rmax = torch.empty(photons.num_data, dtype=_i32, device=dev)
        self.logz = torch.empty(photons.num_data, dtype=_f64, device=dev)

    # -- stages ------------------------------------------------------------
    def slices(self, model):
        """a4 + a5: holographic slices, masked sums, vscale and init."""
        if model.dtype != torch.complex128 or not model.is_contiguous():
            raise ValueError('model must be a contiguous complex128 device tensor')
        s = cur_stream()
        call('rspi_holo_slices', ptr(model), ptr(self.shiftx), ptr(self.shifty), ptr(self.sphere_dia),
            self.n_states0, self.size, ptr(self.bg), ptr(self.sel_pix), self.n_sel,
            ptr(self.holo), ptr(self.msum), s)
        call('rspi_vscale_init', ptr(self.msum), self.n_states0, ptr(self.ph.powder), ptr(self.sel_pix), self.n_sel,
            ptr(self.vscale), ptr(self.init), s)

    def rot_slices(self, r0, r1, out=None):
        """a6: rotated log-slices of rows [r0, r1) into ``out`` (or the chunk buffer)."""
        out = self.lsl if out is None else out
        call('rspi_rot_log_slices', ptr(self.holo), self.n_states0, self.num_rot, ptr(self.rot_cs), self.size,
            ptr(self.bg), ptr(self.sel_pix), self.n_sel, self.p_pad, r0, r1, ptr(out),
            self.slice_code, cur_stream())
        return out

    def loglike(self, r0, r1, lsl=None):
        """a7: likelihood rows [r0, r1); ``lsl`` holds those rows' slices from
        its first row on (default: the chunk buffer)."""
        lsl = self.lsl if lsl is None else lsl
        ll = self.ll
        call('rspi_loglike', ptr(lsl), self.slice_code, self.p_pad, self.num_rot, ptr(self.init),
            ptr(self.ph.scales), ptr(ll['entries']), ptr(ll['row_off']), ptr(ll['order']),
            self.ph.num_data, r0, r1, ptr(self.prob[r0]), self.prob_code, self.ph.num_data,
            self.tile, self.warps, self.n_ctas, cur_stream())

    def run(self, model):
        """Full likelihood matrix ``prob`` for ``model`` (a4-a7)."""
        self.slices(model)
        for r0 in range(0, self.n_rows, self.chunk_rows):
            r1 = min(self.n_rows, r0 + self.chunk_rows)
            self.rot_slices(r0, r1)
            self.loglike(r0, r1)
        return self.prob

    def reduce(self):
        """a8 + a9: per-frame max, first-index argmax and log-sum-exp."""
        call('rspi_frame_reduce', ptr(self.prob), self.prob_code, self.n_rows, self.ph.num_data, ptr(self.maxll),
            ptr(self.rmax), ptr(self.logz), cur_stream())
        return self.maxll, self.rmax, self.logz


class MStep:
    """MaxLP pattern search of every phaser pixel (a11-a14)."""

    def __init__(self, photons, size, num_iter=10):
        self.lib = load()
        self.ph = photons
        self.device = dev = photons.device
        self.size = int(size)
        self.num_iter = int(num_iter)
        g = geometry.phaser_pixels(self.size)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype='i4')).to(dev)  # noqa: E731
        self.mask_idx = t(g['mask_idx'])
        self.n_hist_rows = int(g['n_rows'])
        self.ring, self.ring_rows = t(g['ring']), t(g['ring_rows'])
        self.main, self.main_rows = t(g['main']), t(g['main_rows'])
        self.n_ring, self.n_main = int(g['ring'].size), int(g['main'].size)
        self.rescales = torch.empty(max(1, self.n_ring), dtype=_f64, device=dev)
        self.rescale = torch.empty(1, dtype=_f64, device=dev)
        self.fstate = torch.empty(photons.num_data, dtype=_i32, device=dev)
        self.frot = torch.empty(photons.num_data, dtype=_i32, device=dev)
        self.hist = None
        self.nstate = None

    def frame_params_from_rmax(self, rmax, num_rot, n_ref):
        """fstate / frot / nstate from the E-step argmax (emc.py:218-224)."""
        if self.nstate is None or self.nstate.numel() != n_ref:
            self.nstate = torch.empty(n_ref, dtype=_i32, device=self.device)
        call('rspi_maxlp_frame_params', ptr(rmax), self.ph.num_data, int(num_rot), int(n_ref), ptr(self.fstate),
            ptr(self.frot), ptr(self.nstate), ptr(self.ph.err.t), cur_stream())

    def set_frame_params(self, fstate, frot, nstate):
        self.fstate, self.frot, self.nstate = fstate, frot, nstate

    def run(self, fconv, ref_params, rot_cs):
        """Update ``fconv`` (complex128 device tensor) in place."""
        n_ref = int(ref_params.shape[0])
        need = self.n_hist_rows * n_ref
        if self.hist is None or self.hist.numel() < need:
            self.hist = torch.empty(max(1, need), dtype=_i32, device=self.device)
        hist = self.hist[:max(1, need)]
        hist.zero_()
        s = cur_stream()
        ph = self.ph
        call('rspi_maxlp_histogram', ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum), ptr(ph.multi_accum),
            ptr(ph.place_ones), ptr(ph.place_multi), ptr(ph.count_multi), ph.num_data,
            ptr(self.fstate), ptr(self.frot), ptr(rot_cs), self.size, ptr(self.mask_idx),
            self.n_hist_rows, n_ref, ptr(hist), ptr(ph.err.t), s)
        call('rspi_maxlp_pattern', ptr(fconv), ptr(self.ring), ptr(self.ring_rows), self.n_ring, ptr(hist), n_ref,
            ptr(self.nstate), ph.num_data, ptr(ref_params), self.size, 0, None,
            self.num_iter, ptr(self.rescales), s)
        if self.n_ring > 0:
            call('rspi_mean', ptr(self.rescales), self.n_ring, ptr(self.rescale), s)
        else:
            self.rescale.fill_(float('nan'))   # np.mean of an empty ring
        call('rspi_maxlp_pattern', ptr(fconv), ptr(self.main), ptr(self.main_rows), self.n_main, ptr(hist), n_ref,
            ptr(self.nstate), ph.num_data, ptr(ref_params), self.size, 1, ptr(self.rescale),
            self.num_iter, None, s)
        return fconv
