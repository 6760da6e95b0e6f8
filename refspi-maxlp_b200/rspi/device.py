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
INT32_MAX = 2 ** 31 - 1
QUAD4_WINDOW = 512   # frames ordered by group counts within such windows (four-row quads)
QUAD4_SMEM = 227 * 1024 - 1024   # shared bytes of the four-row tile (kernel limit)
QUAD4_MAX_PARTS = 4              # column parts of the four-row tile
QUAD4_COLS = (QUAD4_SMEM // 16 - 8) // 8 * 8   # most columns of one part
SETS_SWEEPS = 4                  # pair sweeps of the frame grouping (rspi_sets_group)
PIXEL_MAP_MAX_ROT = 1024         # rotation tables the M-step's pixel map serves
PIXEL_MAP_MAX = 1 << 26          # (rotation, detector pixel) entries of that map


def quad4_parts(p_row, parts=None):
    """(parts, columns per part) of the four-row frame-quad tile for a slice
    row of ``p_row`` columns (the last 32 zero): the fewest parts (or
    ``parts``) of a multiple of 8 columns covering the ``p_row - 32``
    likelihood columns whose four FP32 rows, 16 bytes a column plus 8 zero
    columns, fit the kernel's shared memory."""
    pz = int(p_row) - 32
    parts = int(parts) if parts else max(1, -(-pz // QUAD4_COLS))
    part_w = max(8, (-(-pz // parts) + 7) // 8 * 8)
    if parts < 1 or parts > QUAD4_MAX_PARTS or part_w > QUAD4_COLS:
        raise ValueError('%d likelihood columns need more than %d column parts of the '
                         'four-row tile' % (pz, QUAD4_MAX_PARTS))
    return parts, part_w


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
                 need_scaling=False, device=None, frames=None):
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
        self._dense = None
        self.frames = None
        if frames is not None:
            frames = np.ascontiguousarray(frames, dtype=np.uint16)
            if frames.shape != (n, self.num_pix):
                raise ValueError('frames must be (num_data, num_pix) = (%d, %d)' % (n, self.num_pix))
            # raw 16-bit counts (torch has no general uint16 arithmetic; the
            # kernels read them as unsigned short)
            self.frames = torch.from_numpy(frames.view(np.int16)).to(self.device)

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


    def dense_entries(self, sel_pix, n_sel, k_pad, kind='bf16'):
        """Count operands of the dense frames over the likelihood pixels
        (built once per kind): ``kind='bf16'``: BF16 digits ``a0`` = K & 255,
        ``a1`` = K - a0 when some K > 255; ``kind='i8'``: u8 counts ``a0``
        (``kmax`` > 255 means they were clamped and cannot be used)."""
        key = (int(k_pad), sel_pix.data_ptr(), kind)
        if self._dense is not None and self._dense['key'] == key:
            return self._dense
        if self.frames is None:
            raise ValueError('the dense form needs dense frames (a photons file with "frames")')
        n, dev, s = self.num_data, self.device, cur_stream()
        kmax = torch.zeros(1, dtype=_i32, device=dev)
        if kind == 'i8':
            a0 = torch.empty((n, k_pad), dtype=torch.uint8, device=dev)
            call('rspi_dense_frames_u8', ptr(self.frames), n, self.num_pix, ptr(sel_pix), n_sel,
                 k_pad, ptr(a0), ptr(kmax), s)
            self._dense = dict(key=key, a0=a0, a1=None, kmax=int(kmax.item()))
            return self._dense
        a0 = torch.empty((n, k_pad), dtype=torch.bfloat16, device=dev)
        call('rspi_dense_frames', ptr(self.frames), n, self.num_pix, ptr(sel_pix), n_sel, k_pad,
             ptr(a0), None, ptr(kmax), s)
        a1 = None
        if int(kmax.item()) > 255:
            a1 = torch.empty_like(a0)
            call('rspi_dense_frames', ptr(self.frames), n, self.num_pix, ptr(sel_pix), n_sel, k_pad,
                 ptr(a0), ptr(a1), ptr(kmax), s)
        self._dense = dict(key=key, a0=a0, a1=a1, kmax=int(kmax.item()))
        return self._dense

    def ll16_entries(self, pix2sel, p_zero):
        """16-bit count-expanded entries for the FP32 screening pass."""
        key = (int(p_zero), pix2sel.data_ptr())
        if getattr(self, '_ll16', None) is not None and self._ll16['key'] == key:
            return self._ll16
        n, dev, s = self.num_data, self.device, cur_stream()
        rows = torch.empty(n, dtype=_i32, device=dev)
        args = (ptr(self.ones), ptr(self.multi), ptr(self.ones_accum), ptr(self.multi_accum),
                ptr(self.place_ones), ptr(self.place_multi), ptr(self.count_multi), ptr(pix2sel),
                self.num_pix, n, int(p_zero))
        call('rspi_ll16_entry_rows', *args, ptr(rows), ptr(self.err.t), s)
        row_off = torch.empty(n + 1, dtype=_i64, device=dev)
        call('rspi_scan_rows', ptr(rows), n, ptr(row_off), s)
        self.err.check('16-bit entry rows')
        total = int(row_off[-1].item())
        entries = torch.empty(max(2, total) * 32, dtype=torch.int16, device=dev)
        call('rspi_ll16_entry_fill', *args, ptr(row_off), ptr(entries), s)
        order = torch.argsort(rows, descending=True, stable=True).to(_i32)
        mx = torch.zeros(1, dtype=_i32, device=dev)
        call('rspi_entries16_check', ptr(entries), total * 32, ptr(mx), s)
        if int(mx.item()) >= int(p_zero) + 32:
            raise RuntimeError('16-bit entry index %d outside the slice row' % int(mx.item()))
        self._ll16 = dict(key=key, frame_rows=rows, row_off=row_off, entries=entries,
                          order=order, total_rows=total)
        return self._ll16

class EStep:
    """Likelihood of every frame in every (shift, diameter, rotation) state.

    ``form='fp64'``: FP64 rotated slices and FP64 likelihood matrix (the
    plain form).  ``form='screen'``: FP32 slices and likelihood matrix from
    the 16-bit photon entries, then FP64 rescoring of every state within
    ``delta`` (+ the FP32 error bound) of each frame's maximum, which gives
    the same argmax, maximum and log-sum-exp as the FP64 form (the chosen
    form).  ``form='dense'`` (frames stored densely, high fluence): the
    likelihood is a tensor-core GEMM over every likelihood pixel, either
    ``dense_gemm='i8'`` (u8 counts x fixed-point log-slice digits, exact
    int32 accumulation: error <= 2^-22 photons per frame) or
    ``dense_gemm='bf16'`` (BF16 count digits x BF16 hi + lo log-slices, FP32
    accumulation); ``'auto'`` takes i8 when every count is below 256.  With
    ``dense_rescore`` the candidates within delta + 2 eps of each frame's
    maximum are rescored in FP64 as in the screened form; without it the
    GEMM values are final (FP64 log-sum-exp over them).

    ``kernel`` (the likelihood kernel): for the screened form ``sets`` (the
    default: frames 32 at a time, one lane per frame, a bank-conflict-free
    step schedule; likelihood columns in set order, ``frame_prob()`` gives
    frame order), ``quad4`` (four frames per warp) or ``stream``; for the
    FP64 form ``stream`` (default) or ``dynamic``.  ``slice_math``: ``fp32``
    (the frame-set kernel's default, for it only) interpolates and logs the
    slices in FP32 within a bound that the candidate threshold covers;
    ``fp64`` computes them in FP64 and stores them in FP32.  ``set_order``
    (frame-set kernel): ``grouped`` (default) picks each quarter warp's
    eight frames among 256 of alike photon count so that their bank-class
    totals stay close to their mean (``rspi_sets_group``); ``rank`` takes
    them in rank order.
    """

    def __init__(self, photons, size, num_rot, shiftx, shifty, sphere_dia, probmask, bg,
                 form='fp64', states_per_tile=None, warps=32, n_ctas=0,
                 slice_budget_bytes=8 << 30, delta=20., cand_per_frame=None, kernel=None,
                 n_modes=1, dense_gemm='auto', dense_rescore=True, screen_parts=None,
                 slice_math=None, set_order='grouped'):
        if form not in ('fp64', 'screen', 'dense'):
            raise ValueError('form must be fp64, screen or dense')
        if kernel is None:   # default likelihood kernel of each form
            kernel = 'sets' if form == 'screen' else 'stream'
        kernels = {'fp64': ('stream', 'dynamic'), 'screen': ('stream', 'quad4', 'sets'),
                   'dense': ('stream', 'tcgen05')}[form]
        if kernel not in kernels:
            raise ValueError('the %s form takes the kernels %s' % (form, ', '.join(kernels)))
        self.screen_parts = None if screen_parts is None else int(screen_parts)
        if slice_math is None:
            slice_math = 'fp32' if kernel == 'sets' else 'fp64'
        if slice_math not in ('fp64', 'fp32'):
            raise ValueError('slice_math must be fp64 or fp32')
        if slice_math == 'fp32' and kernel != 'sets':
            raise ValueError('FP32 slice arithmetic is for the frame-set kernel')
        self.slice_math = slice_math
        if set_order not in ('grouped', 'rank'):
            raise ValueError('set_order must be grouped or rank')
        self.set_order = set_order
        self.kernel = kernel
        self.lib = load()
        self.form = form
        self.ph = photons
        self.device = dev = photons.device
        self.size, self.num_rot = int(size), int(num_rot)
        # n_modes models share the (shift, diameter) grid: state m*S0 + s,
        # likelihood row (m*S0 + s)*num_rot + j
        self.n_modes = int(n_modes)
        if self.n_modes < 1:
            raise ValueError('n_modes must be at least 1')
        self.n_grid = int(np.asarray(shiftx).size)
        self.n_states0 = self.n_grid * self.n_modes
        self.n_rows = self.n_states0 * self.num_rot
        n = photons.num_data
        sel, pix2sel, p_pad = geometry.sel_pixels(probmask)
        self.n_sel, self.p_pad = sel.size, p_pad
        t = lambda a, dt=_f64: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        # a detector without likelihood pixels still passes a valid pointer
        self.sel_pix = t(sel if sel.size else np.zeros(1, 'i4'), _i32)
        self.pix2sel = t(pix2sel, _i32)
        self.shiftx, self.shifty, self.sphere_dia = t(shiftx), t(shifty), t(sphere_dia)
        self.rot_cs = t(geometry.emc_rotation_table(self.num_rot))
        self.bg = t(np.asarray(bg, dtype='f8').ravel())
        self.ll = photons.ll_entries(self.pix2sel, self.p_pad)
        self.col_of_frame, self.frame_of_col, self.n_cols = None, None, n
        self.holo_quads32 = None
        if form == 'dense':
            self._init_dense(photons, slice_budget_bytes, delta, cand_per_frame, dense_gemm,
                             dense_rescore)
            return
        if form == 'fp64':
            self.slice_code, self.prob_code, self.p_row = 1, 1, self.p_pad
        else:
            # FP32 slices; 32 zero columns after the likelihood columns for
            # the padding slots of the 16-bit entries
            self.slice_code, self.prob_code = 0, 0
            self.p_row = self.p_pad + 32
            if self.p_row > 65536:
                raise ValueError('screened form needs at most 65504 likelihood pixels')
            self.ll16 = photons.ll16_entries(self.pix2sel, self.p_row - 32)
            self.delta = float(delta)
        self.slice_torch = {0: torch.float32, 1: _f64}[self.slice_code]
        self.prob_torch = torch.float32 if self.prob_code == 0 else _f64
        if kernel in ('quad4', 'sets'):
            tmax = 4                 # four rows per tile over column parts
            if self.p_row - 32 > QUAD4_MAX_PARTS * QUAD4_COLS:
                raise ValueError('%d likelihood columns exceed the four-row tile' % self.n_sel)
        else:
            tmax = self.lib.rspi_loglike_max_tile(self.p_row, self.slice_code)
        if tmax == 0:
            raise ValueError('a %d-pixel likelihood slice does not fit in shared memory' % self.n_sel)
        self.tile = int(states_per_tile or tmax)
        if self.tile > tmax:
            raise ValueError('states_per_tile %d exceeds the shared-memory limit %d' % (self.tile, tmax))
        if kernel in ('quad4', 'sets') and self.tile != 4:
            raise ValueError('the four-row %s kernel takes 4 states per tile' % kernel)
        self.warps, self.n_ctas = int(warps), int(n_ctas)
        # column order of the likelihood matrix: frame order, except for the
        # frame-set kernel (column 32 s + l = frame set_frames[32 s + l])
        self.wide = None
        if kernel == 'quad4':
            self.wide = self._quad4_entries()
        elif kernel == 'sets':
            self.wide = self._sets_entries()
            self.col_of_frame = self.wide['col_of_frame']
            self.frame_of_col = self.wide['set_frames']
            self.n_cols = self.wide['n_sets'] * 32
            self.frame_max = torch.zeros(self.n_cols, dtype=_i64, device=dev)
            self.cand_slot = torch.empty(n * 32, dtype=_i32, device=dev)
        # FP32 copy of the four bilinear corners for the FP32 slice arithmetic
        self.holo_quads32 = torch.empty((self.n_states0, self.size ** 2, 4),
                                        dtype=torch.float32, device=dev) \
            if self.slice_math == 'fp32' else None
        self._eps_key, self.row_off_eps = None, None
        esz = {0: 4, 1: 8, 2: 2}[self.slice_code]
        # slice bytes per likelihood row (the frame-set layout holds the
        # column parts without the 32 zero columns)
        row_bytes = (self.wide['n_parts'] * self.wide['part_w'] * 4 if kernel == 'sets'
                     else self.p_row * esz)
        rows = max(self.tile, (slice_budget_bytes // row_bytes) // self.tile * self.tile)
        self.chunk_rows = int(min(self.n_rows, rows))
        self.holo = torch.empty((self.n_states0, self.size ** 2), dtype=_f64, device=dev)
        # (w[p], w[p + 1]) pairs: the slice kernel's bilinear rows as 16-byte loads
        self.holo_pairs = torch.empty((self.n_states0, self.size ** 2, 2), dtype=_f64,
                                      device=dev)
        self.msum = torch.empty(self.n_states0, dtype=_f64, device=dev)
        self.vscale = torch.empty(1, dtype=_f64, device=dev)
        self.init = torch.empty(self.n_states0, dtype=_f64, device=dev)
        if kernel == 'sets':
            # tiles of four rows x parts x part_w float4 columns
            tiles = (self.chunk_rows + 3) // 4
            self.lsl = torch.empty(tiles * self.wide['n_parts'] * self.wide['part_w'] * 4,
                                   dtype=torch.float32, device=dev)
        else:
            self.lsl = torch.empty((self.chunk_rows, self.p_row), dtype=self.slice_torch,
                                   device=dev)
        self.prob = torch.empty((self.n_rows, self.n_cols), dtype=self.prob_torch, device=dev)
        self.maxll = torch.empty(n, dtype=_f64, device=dev)
        self.rmax = torch.empty(n, dtype=_i32, device=dev)
        self.logz = torch.empty(n, dtype=_f64, device=dev)
        if form == 'screen':
            self.lmax = torch.zeros(1, dtype=torch.float32, device=dev)
            self.max32 = torch.empty(n, dtype=_f64, device=dev)
            self.rmax32 = torch.empty(n, dtype=_i32, device=dev)
            self.cnt_part = torch.empty(n * 32, dtype=_i32, device=dev)
            self.cand_n = torch.empty(n, dtype=_i32, device=dev)
            self.noncand = torch.empty(n, dtype=_f64, device=dev)
            self.thr = torch.empty(n, dtype=_f64, device=dev)
            self.cand_off = torch.empty(n + 1, dtype=_i64, device=dev)
            self.row_cnt = torch.empty(self.n_rows, dtype=_i32, device=dev)
            self.row_cand_off = torch.empty(self.n_rows + 1, dtype=_i64, device=dev)
            self._alloc_row_scratch()
            per = int(cand_per_frame) if cand_per_frame else min(self.n_rows, 8192)
            self._alloc_candidates(max(1024, per * n))
        self.check_capacity = True
        self.ll_events = None   # list -> (start, end, rows) CUDA events around each launch

    def _init_dense(self, photons, slice_budget_bytes, delta, cand_per_frame, dense_gemm,
                    dense_rescore):
        dev, n = self.device, photons.num_data
        if dense_gemm not in ('auto', 'i8', 'bf16'):
            raise ValueError('dense_gemm must be auto, i8 or bf16')
        self.kernel = 'tcgen05'
        self.slice_code, self.prob_code = 2, 0           # 4 bytes of slice operands per value
        self.k_pad = (self.n_sel + 127) // 128 * 128
        self.p_row = self.k_pad
        self.rescore = bool(dense_rescore)
        phot_max = int(self.ll['frame_sel_photons'].max().item())
        gemm = dense_gemm
        if gemm in ('auto', 'i8'):
            dn = photons.dense_entries(self.sel_pix, self.n_sel, self.k_pad, 'i8')
            fits = dn['kmax'] <= 255 and phot_max * 255 < 2 ** 31
            if gemm == 'i8' and not fits:
                raise ValueError('the exact integer GEMM needs counts below 256 and fewer than '
                                 '8.4e6 photons per frame on the likelihood pixels')
            gemm = 'i8' if fits else 'bf16'
        self.dense_gemm = gemm
        self.dense = photons.dense_entries(self.sel_pix, self.n_sel, self.k_pad, gemm)
        self.n_digits = 2 if self.dense['a1'] is not None else 1
        self.delta = float(delta)
        self.slice_torch, self.prob_torch = torch.bfloat16, torch.float32
        self.tile = 128
        rows = max(128, (slice_budget_bytes // (self.k_pad * 4)) // 128 * 128)
        self.chunk_rows = int(min(self.n_rows, rows))
        npix = self.size ** 2
        self.holo = torch.empty((self.n_states0, npix), dtype=_f64, device=dev)
        self.msum = torch.empty(self.n_states0, dtype=_f64, device=dev)
        self.vscale = torch.empty(1, dtype=_f64, device=dev)
        self.init = torch.empty(self.n_states0, dtype=_f64, device=dev)
        if gemm == 'i8':
            self.lsl = torch.empty((4, self.chunk_rows, self.k_pad), dtype=torch.uint8, device=dev)
        else:
            self.lsl_hi = torch.empty((self.chunk_rows, self.k_pad), dtype=torch.bfloat16,
                                      device=dev)
            self.lsl_lo = torch.empty_like(self.lsl_hi)
            self.lsl = self.lsl_hi
        self.prob = torch.empty((self.n_rows, n), dtype=torch.float32, device=dev)
        self.maxll = torch.empty(n, dtype=_f64, device=dev)
        self.rmax = torch.empty(n, dtype=_i32, device=dev)
        self.logz = torch.empty(n, dtype=_f64, device=dev)
        self.lmax = torch.zeros(1, dtype=torch.float32, device=dev)
        self.max32 = torch.empty(n, dtype=_f64, device=dev)
        self.rmax32 = torch.empty(n, dtype=_i32, device=dev)
        self.cnt_part = torch.empty(n * 32, dtype=_i32, device=dev)
        self.cand_n = torch.empty(n, dtype=_i32, device=dev)
        self.noncand = torch.empty(n, dtype=_f64, device=dev)
        self.thr = torch.empty(n, dtype=_f64, device=dev)
        self.cand_off = torch.empty(n + 1, dtype=_i64, device=dev)
        self.row_cnt = torch.empty(self.n_rows, dtype=_i32, device=dev)
        self.row_cand_off = torch.empty(self.n_rows + 1, dtype=_i64, device=dev)
        self._alloc_row_scratch()
        # Error bound of the GEMM value.  The candidate threshold's eps_d is
        # 2^-24 ((rows + 8) photons lmax + |max| + delta + 1) (+ 1e-9 photons
        # lmax).  i8: the quantisation bound 2^-22 photons is rows = 0 with
        # lmax = 1/2.  bf16: 2^-16 relative from the hi + lo split (256 steps
        # of 2^-24) plus 2 x 2^-24 for each of the n_steps tensor-core
        # accumulations (a rounding or truncating FP32 adder), as the same
        # per-frame row count for every frame, with lmax the slices' max |L|.
        if gemm == 'i8':
            self.eq_rows = 0
            self.lmax_eps = torch.full((1,), 0.5, dtype=torch.float32, device=dev)
        else:
            n_steps = (self.k_pad // 16) * self.n_digits * 2
            self.eq_rows = 256 + 2 * n_steps
            self.lmax_eps = self.lmax
        self.eq_row_off = torch.arange(n + 1, dtype=_i64, device=dev) * self.eq_rows
        per = int(cand_per_frame) if cand_per_frame else min(self.n_rows, 8192)
        self._alloc_candidates(max(1024, per * n))
        self.check_capacity = True
        self.ll_events = None

    def parts(self):
        """Column parts of the four-row kernels' tile (None for the others)."""
        return None if self.wide is None else int(self.wide['n_parts'])

    def configure(self, warps=None, screen_parts=None, tile=None):
        """Change the likelihood kernel's tiling -- warps per CTA, the column
        parts of the four-row kernels, the rows per tile of the streaming
        kernels -- rebuilding the entries and buffers that depend on it.
        The FP64-rescored results do not depend on the tiling."""
        if warps is not None:
            self.warps = int(warps)
        if tile is not None and int(tile) != self.tile:
            if self.kernel in ('quad4', 'sets'):
                raise ValueError('the four-row kernels take 4 states per tile')
            tmax = self.lib.rspi_loglike_max_tile(self.p_row, self.slice_code)
            if not 1 <= int(tile) <= tmax:
                raise ValueError('states_per_tile %d outside 1..%d' % (int(tile), tmax))
            self.tile = int(tile)
        if screen_parts is not None and self.kernel in ('quad4', 'sets') and \
                int(screen_parts) != self.parts():
            self.screen_parts = int(screen_parts)
            if self.kernel == 'quad4':
                self.wide = self._quad4_entries()
            else:
                self.wide = self._sets_entries()
                self.col_of_frame = self.wide['col_of_frame']
                self.frame_of_col = self.wide['set_frames']
                need = ((self.chunk_rows + 3) // 4) * self.wide['n_parts'] * \
                    self.wide['part_w'] * 4
                if self.lsl.numel() < need:
                    self.lsl = torch.empty(need, dtype=torch.float32, device=self.device)
            self._eps_key = None

    def _quad4_parts(self):
        """Column parts of the four-row tile (``quad4_parts``), or
        ``screen_parts`` parts."""
        return quad4_parts(self.p_row, self.screen_parts)

    def _quad4_entries(self):
        """Entries of the four-row frame-quad kernel: frames ordered within
        each window of QUAD4_WINDOW by decreasing group counts, part 0 first,
        and taken four at a time; per (quad, column part) the largest of
        its frames' group counts, group ranges part-major; lane j of a
        sub-frame holds the photons of local column class j (mod 8); one
        FP32 running sum per (CTA, row, frame slot) when there are several
        parts."""
        l16, n, dev, s = self.ll16, self.ph.num_data, self.device, cur_stream()
        pz = self.p_row - 32
        parts, part_w = self._quad4_parts()
        ng = torch.empty(n * parts, dtype=_i32, device=dev)
        call('rspi_quad4_entry_groups', ptr(l16['entries']), ptr(l16['row_off']), n, pz, parts,
             part_w, ptr(ng), s)
        ngp = ng.view(n, parts).to(_i64)
        # within each window, frames in decreasing (part 0, part 1, ...) group
        # counts: a quad's frames then need alike counts in every part
        order = torch.arange(n, device=dev, dtype=_i64)
        for h in reversed(range(parts)):
            order = order[torch.argsort(-ngp[order, h], stable=True)]
        order = order[torch.argsort(order // QUAD4_WINDOW, stable=True)].to(_i32)
        nq = (n + 3) // 4
        set_frames = torch.full((4 * nq,), -1, dtype=_i32, device=dev)
        set_frames[:n] = order
        set_slot = torch.empty(n, dtype=_i32, device=dev)
        set_slot[order.long()] = torch.arange(n, dtype=_i32, device=dev)
        ngs = torch.zeros((4 * nq, parts), dtype=_i64, device=dev)
        ngs[:n] = ngp[order.long()]
        sng = ngs.view(nq, 4, parts).amax(1)                       # (quad, part)
        flat = sng.t().contiguous().view(-1).to(_i32)             # part-major
        soff = torch.empty(parts * nq + 1, dtype=_i64, device=dev)
        call('rspi_scan_rows', ptr(flat), parts * nq, ptr(soff), s)
        total = int(soff[-1].item())
        narrow = torch.empty(max(1, total) * 128, dtype=torch.int16, device=dev)
        call('rspi_quad4_entry_fill', ptr(l16['entries']), ptr(l16['row_off']), n, pz, parts,
             part_w, ptr(set_slot), ptr(soff), nq, total, ptr(narrow), s)
        ps, ps_ctas = None, 0
        if parts > 1:
            ps_ctas = self.n_ctas if self.n_ctas > 0 else \
                torch.cuda.get_device_properties(dev).multi_processor_count
            nfl = self.lib.rspi_quad4_part_sums_floats(nq, ps_ctas)
            ps = torch.empty(nfl, dtype=torch.float32, device=dev)
        return dict(entries=narrow, group_off=soff, total_groups=total, tile=4, banked=True,
                    narrow=True, pairs=True, frames_per=4, quad4=True, pair_frames=set_frames,
                    n_pairs=nq, frame_groups=sng.amax(1)[(set_slot // 4).long()],
                    n_parts=parts, part_w=part_w, part_sums=ps, part_sums_ctas=ps_ctas)

    def _sets_entries(self):
        """Entries of the frame-set kernel: frames in decreasing order of
        their likelihood-pixel photons, grouped per 256 ranks into quarter
        warps whose class totals stay close to their mean and quarters of
        alike cost four to a set (``set_order='grouped'``), or lane 8 p + f
        of set s the frame of rank 32 s + p + 4 f (``'rank'``).  Per (set,
        column part) a step schedule
        in which a quarter warp's eight lanes read eight distinct bank
        classes (rspi_sets_steps / rspi_sets_fill); one FP32 running sum per
        (CTA, column) between parts when there are several."""
        l16, n, dev, s = self.ll16, self.ph.num_data, self.device, cur_stream()
        pz = self.p_row - 32
        parts, part_w = self._quad4_parts()
        counts = torch.empty(n * 32, dtype=_i32, device=dev)
        call('rspi_sets_counts', ptr(l16['entries']), ptr(l16['row_off']), n, pz, parts, part_w,
             ptr(counts), s)
        tot = self.ll['frame_sel_photons']
        order = torch.argsort(-tot, stable=True)
        n_sets = (n + 31) // 32
        k = torch.arange(n_sets * 32, device=dev, dtype=_i64)
        if self.set_order == 'grouped':
            set_frames = torch.empty(n_sets * 32, dtype=_i32, device=dev)
            call('rspi_sets_group', ptr(counts), ptr(order.to(_i32)), n, parts, SETS_SWEEPS,
                 ptr(set_frames), ptr(self.ph.err.t), s)
            self.ph.err.check('frame grouping')
        else:
            lane = k % 32
            src = (k - lane) + (lane // 8) + 4 * (lane % 8)
            set_frames = torch.where(src < n, order[src.clamp(max=n - 1)],
                                     torch.full_like(src, -1)).to(_i32)
        col_of_frame = torch.empty(n, dtype=_i32, device=dev)
        real = set_frames >= 0
        col_of_frame[set_frames[real].long()] = k[real].to(_i32)
        groups = torch.empty(parts * n_sets, dtype=_i32, device=dev)
        qgroups = torch.empty(parts * n_sets * 4, dtype=_i32, device=dev)
        call('rspi_sets_steps', ptr(counts), ptr(set_frames), n_sets, parts, ptr(groups),
             ptr(qgroups), s)
        goff = torch.empty(parts * n_sets + 1, dtype=_i64, device=dev)
        call('rspi_scan_rows', ptr(groups), parts * n_sets, ptr(goff), s)
        total = int(goff[-1].item())
        # every slot starts at the zero column part_w (class 0), a valid index
        entries = torch.full((max(1, total) * 128,), part_w, dtype=torch.int16, device=dev)
        call('rspi_sets_fill', ptr(l16['entries']), ptr(l16['row_off']), pz, parts, part_w,
             ptr(counts), ptr(set_frames), n_sets, ptr(goff), ptr(entries), ptr(self.ph.err.t),
             s)
        self.ph.err.check('frame-set entries')
        bad = torch.zeros(1, dtype=_i32, device=dev)
        call('rspi_sets_entries_check', ptr(entries), max(1, total) * 128, part_w, ptr(bad), s)
        if int(bad.item()) != 0:
            raise RuntimeError('%d frame-set entries outside the staged part' % int(bad.item()))
        # each frame's FP32 summation length for the candidate threshold:
        # ceil(G / 2) accumulator steps of its set's largest part (the +3 of
        # the group tree and the final add are within the threshold's +8)
        g = groups.view(parts, n_sets).to(_i64)
        per_set = ((g + 1) // 2).amax(0)
        frame_groups = torch.zeros(n, dtype=_i64, device=dev)
        frame_groups[set_frames[real].long()] = per_set[(k[real] // 32)]
        ps, ps_ctas = None, 0
        if parts > 1:
            ps_ctas = self.n_ctas if self.n_ctas > 0 else \
                torch.cuda.get_device_properties(dev).multi_processor_count
            ps = torch.empty(self.lib.rspi_sets_part_sums_floats(n_sets, ps_ctas),
                             dtype=torch.float32, device=dev)
        return dict(entries=entries, group_off=goff, quarter_groups=qgroups,
                    total_groups=total, tile=4, sets=True,
                    set_frames=set_frames, col_of_frame=col_of_frame, n_sets=n_sets,
                    frame_groups=frame_groups, n_parts=parts, part_w=part_w, part_sums=ps,
                    part_sums_ctas=ps_ctas, counts=counts)

    def _eps_rows(self):
        """Prefix sums of each frame's FP32 summation length for the
        candidate threshold's eps_d (the 'rows' of 2^-24 (rows + 8) photons
        lmax): the frame's 16-bit entry rows, or the summation length of the
        kernel's entry layout when that is longer."""
        key = (self.kernel, None if self.wide is None else self.wide['entries'].data_ptr())
        if key != self._eps_key:
            ro = self.ll16['row_off']
            rows = ro[1:] - ro[:-1]
            if self.wide is not None:
                rows = torch.maximum(rows, self.wide['frame_groups'].to(_i64))
            if self.slice_math == 'fp32':
                rows = rows + 23
            self.row_off_eps = torch.cat([torch.zeros(1, dtype=_i64, device=self.device),
                                          torch.cumsum(rows, 0)])
            self._eps_key = key
        return self.row_off_eps

    def _alloc_row_scratch(self):
        """Global rows for FP64 rescoring when a row exceeds shared memory
        (one per SM; none otherwise)."""
        self.row_scratch, self.scratch_rows = None, 0
        if self.p_pad * 8 > 220 * 1024:
            sms = torch.cuda.get_device_properties(self.device).multi_processor_count
            self.scratch_rows = int(sms)
            self.row_scratch = torch.empty((sms, self.p_pad), dtype=_f64, device=self.device)

    def _alloc_candidates(self, cap):
        dev = self.device
        self.capacity = int(cap)
        self.cand_d = torch.empty(self.capacity, dtype=_i32, device=dev)
        self.cand_r = torch.empty(self.capacity, dtype=_i32, device=dev)
        self.cand_ll = torch.empty(self.capacity, dtype=_f64, device=dev)
        self.row_cand = torch.empty(self.capacity, dtype=_i32, device=dev)

    # -- stages ------------------------------------------------------------
    def slices(self, model):
        """a4 + a5: holographic slices, masked sums, vscale and init."""
        npix = self.size ** 2
        if model.dtype != torch.complex128 or not model.is_contiguous() or \
                model.numel() != self.n_modes * npix:
            raise ValueError('model must be a contiguous complex128 device tensor of %d x %d '
                             'pixels' % (self.n_modes, npix))
        s = cur_stream()
        flat = model.view(-1)
        for m in range(self.n_modes):
            g0 = m * self.n_grid
            call('rspi_holo_slices', ptr(flat[m * npix:]), ptr(self.shiftx), ptr(self.shifty),
                 ptr(self.sphere_dia), self.n_grid, self.size, ptr(self.bg), ptr(self.sel_pix),
                 self.n_sel, ptr(self.holo[g0]), ptr(self.msum[g0:]), s)
        call('rspi_vscale_init', ptr(self.msum), self.n_states0, ptr(self.ph.powder),
             ptr(self.sel_pix), self.n_sel, ptr(self.vscale), ptr(self.init), s)
        if self.form != 'dense':
            call('rspi_holo_pairs', ptr(self.holo), self.n_states0, self.size,
                 ptr(self.holo_pairs), s)
        if self.form != 'fp64':
            # FP32 slice arithmetic: its per-value error bound 2^-24 (16 + 7|L|)
            # is charged as 23 more summation steps of max(|L|, 1)
            self.lmax.fill_(1. if self.slice_math == 'fp32' else 0.)
        if self.holo_quads32 is not None:
            call('rspi_holo_quads32', ptr(self.holo), self.n_states0, self.size,
                 ptr(self.holo_quads32), s)
        if self.col_of_frame is not None:
            self.frame_max.zero_()

    def rot_slices(self, r0, r1, out=None):
        """a6: rotated log-slices of rows [r0, r1) into ``out`` (or the chunk buffer)."""
        if self.form == 'dense' and self.dense_gemm == 'i8':
            call('rspi_rot_log_fixed', ptr(self.holo), self.n_states0, self.num_rot,
                 ptr(self.rot_cs), self.size, ptr(self.bg), ptr(self.sel_pix), self.n_sel,
                 self.k_pad, r0, r1, self.chunk_rows, ptr(self.lsl), ptr(self.ph.err.t),
                 cur_stream())
            return self.lsl
        if self.form == 'dense':
            call('rspi_rot_log_split', ptr(self.holo), self.n_states0, self.num_rot,
                 ptr(self.rot_cs), self.size, ptr(self.bg), ptr(self.sel_pix), self.n_sel,
                 self.k_pad, r0, r1, ptr(self.lsl_hi), ptr(self.lsl_lo), ptr(self.lmax),
                 cur_stream())
            return self.lsl_hi
        out = self.lsl if out is None else out
        if self.kernel == 'sets':
            w = self.wide
            call('rspi_rot_log_slices_sets', ptr(self.holo_pairs), ptr(self.holo_quads32),
                 self.n_states0, self.num_rot,
                 ptr(self.rot_cs), self.size, ptr(self.bg), ptr(self.sel_pix), self.n_sel,
                 w['n_parts'], w['part_w'], r0, r1, ptr(out), ptr(self.lmax), cur_stream())
            return out
        call('rspi_rot_log_slices_pairs', ptr(self.holo_pairs), self.n_states0, self.num_rot,
             ptr(self.rot_cs), self.size, ptr(self.bg), ptr(self.sel_pix), self.n_sel,
             self.p_row, r0, r1, ptr(out), self.slice_code,
             ptr(self.lmax) if self.form == 'screen' else None, cur_stream())
        return out

    def loglike(self, r0, r1, lsl=None):
        """a7: likelihood rows [r0, r1); ``lsl`` holds those rows' slices from
        its first row on (default: the chunk buffer)."""
        lsl = self.lsl if lsl is None else lsl
        n = self.ph.num_data
        if self.ll_events is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), r1 - r0)
            ev[0].record(torch.cuda.current_stream())
        self._loglike_launch(r0, r1, lsl, n)
        if self.ll_events is not None:
            ev[1].record(torch.cuda.current_stream())
            self.ll_events.append(ev)

    def _loglike_launch(self, r0, r1, lsl, n):
        if self.form == 'dense' and self.dense_gemm == 'i8':
            call('rspi_dense_loglike_i8', ptr(self.dense['a0']), ptr(self.lsl), self.k_pad, n,
                 self.chunk_rows, self.num_rot, r0, r1, ptr(self.init), ptr(self.ph.scales),
                 ptr(self.prob[r0]), n, ptr(self.ph.err.t), cur_stream())
        elif self.form == 'dense':
            dn = self.dense
            call('rspi_dense_loglike', ptr(dn['a0']), ptr(dn['a1']), ptr(self.lsl_hi),
                 ptr(self.lsl_lo), self.k_pad, n, self.chunk_rows, self.num_rot, r0, r1,
                 ptr(self.init), ptr(self.ph.scales), ptr(self.prob[r0]), n, ptr(self.ph.err.t),
                 cur_stream())
        elif self.kernel == 'quad4' and self.form == 'screen':
            w = self.wide
            if w is None or not w.get('quad4') or (w['n_parts'] > 1 and self.n_ctas > 0 and
                                                    self.n_ctas != w['part_sums_ctas']):
                w = self.wide = self._quad4_entries()
            call('rspi_screen_loglike7', ptr(lsl), self.p_row, self.num_rot, ptr(self.init),
                 ptr(self.ph.scales), ptr(w['entries']), ptr(w['group_off']),
                 ptr(w['pair_frames']), w['n_pairs'], w['n_parts'], w['part_w'], r0, r1,
                 ptr(self.prob[r0]), n, ptr(w['part_sums']), w['part_sums_ctas'], self.warps,
                 self.n_ctas, cur_stream())
        elif self.kernel == 'sets':
            w = self.wide
            if w['n_parts'] > 1 and self.n_ctas > 0 and self.n_ctas != w['part_sums_ctas']:
                w = self.wide = self._sets_entries()
            call('rspi_screen_loglike_sets', ptr(lsl), self.num_rot, ptr(self.init),
                 ptr(self.ph.scales), ptr(w['entries']), ptr(w['group_off']),
                 ptr(w['quarter_groups']), ptr(w['set_frames']), w['n_sets'], w['n_parts'],
                 w['part_w'], r0, r1,
                 ptr(self.prob[r0]), self.n_cols, ptr(w['part_sums']), w['part_sums_ctas'],
                 ptr(self.frame_max), self.warps, self.n_ctas, ptr(self.ph.err.t), cur_stream())
        elif self.kernel == 'stream' and self.form == 'screen':
            l16 = self.ll16
            call('rspi_loglike_stream', 0, ptr(lsl), self.p_row, self.num_rot, ptr(self.init),
                 ptr(self.ph.scales), ptr(l16['entries']), ptr(l16['row_off']), n, r0, r1,
                 ptr(self.prob[r0]), n, self.tile, self.warps, self.n_ctas, cur_stream())
        elif self.kernel == 'stream':
            ent = self.ll
            call('rspi_loglike_stream', self.slice_code, ptr(lsl), self.p_row, self.num_rot,
                 ptr(self.init), ptr(self.ph.scales), ptr(ent['entries']), ptr(ent['row_off']),
                 n, r0, r1, ptr(self.prob[r0]), n, self.tile, self.warps, self.n_ctas,
                 cur_stream())
        else:
            ll = self.ll
            call('rspi_loglike', ptr(lsl), self.slice_code, self.p_row, self.num_rot,
                 ptr(self.init), ptr(self.ph.scales), ptr(ll['entries']), ptr(ll['row_off']),
                 ptr(ll['order']), n, r0, r1, ptr(self.prob[r0]), self.prob_code, n, self.tile,
                 self.warps, self.n_ctas, cur_stream())

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
        n = self.ph.num_data
        s = cur_stream()
        if self.form == 'fp64' or (self.form == 'dense' and not self.rescore):
            call('rspi_frame_reduce', ptr(self.prob), self.prob_code, self.n_rows, n,
                 ptr(self.maxll), ptr(self.rmax), ptr(self.logz), s)
            return self.maxll, self.rmax, self.logz
        cols = self.col_of_frame is not None
        if cols:
            # the screening kernel already folded each column's maximum into
            # its key
            call('rspi_frame_max_finalize', ptr(self.frame_max), ptr(self.frame_of_col),
                 self.n_cols, ptr(self.max32), ptr(self.rmax32), s)
        else:
            call('rspi_frame_reduce', ptr(self.prob), 0, self.n_rows, n, ptr(self.max32),
                 ptr(self.rmax32), None, s)
        while True:
            dense = self.form == 'dense'
            rows_eq = self.eq_row_off if dense else self._eps_rows()
            tail = (ptr(self.rmax32), ptr(self.ll['frame_sel_photons']), ptr(rows_eq),
                    ptr(self.lmax_eps if dense else self.lmax), self.delta, ptr(self.cnt_part),
                    ptr(self.cand_n), ptr(self.noncand), ptr(self.thr), ptr(self.cand_off),
                    self.capacity, ptr(self.cand_d), ptr(self.cand_r), ptr(self.ph.err.t), s)
            if cols:
                call('rspi_screen_candidates_cols', ptr(self.prob), self.n_rows, self.n_cols,
                     ptr(self.frame_of_col), n, ptr(self.max32), *tail[:-2],
                     ptr(self.cand_slot), *tail[-2:])
            else:
                call('rspi_screen_candidates', ptr(self.prob), self.n_rows, n, ptr(self.max32),
                     *tail)
            if self.check_capacity:
                total = int(self.cand_off[n].item())
                if total > self.capacity:
                    if total > INT32_MAX:
                        raise RuntimeError('%d screened candidates exceed the int32 candidate '
                                           'index; raise the precision of the screening pass or '
                                           'lower screen_delta' % total)
                    self.ph.err.t.zero_()
                    self._alloc_candidates(min(INT32_MAX, int(total * 1.5) + 1024))
                    continue
                self.n_candidates = total
            break
        head = (ptr(self.cand_d), ptr(self.cand_r), ptr(self.cand_off), n, self.capacity,
                self.n_rows, ptr(self.holo), self.num_rot, ptr(self.rot_cs), self.size,
                ptr(self.bg), ptr(self.sel_pix), self.n_sel, self.p_pad, ptr(self.init),
                ptr(self.ph.scales), ptr(self.ll['entries']), ptr(self.ll['row_off']),
                ptr(self.row_cnt), ptr(self.row_cand_off), ptr(self.row_cand), ptr(self.cand_ll),
                ptr(self.prob))
        tail = (ptr(self.max32), ptr(self.noncand), ptr(self.maxll), ptr(self.rmax),
                ptr(self.logz), ptr(self.row_scratch), self.scratch_rows, s)
        if cols:
            call('rspi_rescore_cols', *head, self.n_cols, ptr(self.col_of_frame), *tail)
        else:
            call('rspi_rescore', *head, *tail)
        return self.maxll, self.rmax, self.logz

    def frame_prob(self):
        """The likelihood matrix with frames in their own order (rows x
        frames, the layout of emc.py's ``prob``): ``prob`` itself, or for the
        frame-set kernel, whose columns are in set order, a reordered copy."""
        if self.col_of_frame is None:
            return self.prob
        return self.prob.index_select(1, self.col_of_frame.long())


class Merge:
    """Posterior-weighted merge into per-(shift, diameter) intensities (a10)."""

    def __init__(self, estep, p_min=1.e-6, pairs_per_frame=16):
        self.es = estep
        self.p_min = float(p_min)
        dev = estep.device
        n0, r, npix = estep.n_states0, estep.num_rot, estep.size ** 2
        self.cov = torch.empty((r, npix), dtype=_f64, device=dev)
        call('rspi_merge_coverage', r, ptr(estep.rot_cs), estep.size, ptr(self.cov), cur_stream())
        self.num = torch.empty((n0, npix), dtype=_f64, device=dev)
        self.den = torch.empty((n0, npix), dtype=_f64, device=dev)
        self.w = torch.empty(n0 * r, dtype=_f64, device=dev)
        self.intens = torch.empty((n0, npix), dtype=_f64, device=dev)
        n = estep.ph.num_data
        if estep.form == 'fp64':
            self.cnt_part = torch.empty(n * 32, dtype=_i32, device=dev)
            self.cnt = torch.empty(n, dtype=_i32, device=dev)
            self.off = torch.empty(n + 1, dtype=_i64, device=dev)
            self._alloc(max(1024, pairs_per_frame * n))

    def _alloc(self, cap):
        dev = self.es.device
        self.capacity = int(cap)
        self.pd = torch.empty(self.capacity, dtype=_i32, device=dev)
        self.pr = torch.empty(self.capacity, dtype=_i32, device=dev)
        self.pll = torch.empty(self.capacity, dtype=_f64, device=dev)

    def run(self):
        """intens (S0 x P) from the current likelihoods and log-sum-exp."""
        es, ph, s = self.es, self.es.ph, cur_stream()
        n = ph.num_data
        if es.form == 'fp64':
            while True:
                call('rspi_posterior_pairs', ptr(es.prob), es.n_rows, n, ptr(es.logz), self.p_min,
                     ptr(self.cnt_part), ptr(self.cnt), ptr(self.off), self.capacity, ptr(self.pd),
                     ptr(self.pr), ptr(self.pll), ptr(ph.err.t), s)
                total = int(self.off[n].item())
                if total <= self.capacity:
                    break
                ph.err.t.zero_()
                self._alloc(int(total * 1.25) + 1024)
            pd, pr, pll, tot, cap = self.pd, self.pr, self.pll, self.off[n:], self.capacity
        else:
            pd, pr, pll, tot, cap = es.cand_d, es.cand_r, es.cand_ll, es.cand_off[n:], es.capacity
        call('rspi_merge', ptr(pd), ptr(pr), ptr(pll), ptr(tot), cap, ptr(es.logz), self.p_min,
             ptr(ph.scales), ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum), ptr(ph.multi_accum),
             ptr(ph.place_ones), ptr(ph.place_multi), ptr(ph.count_multi), es.n_states0,
             es.num_rot, ptr(es.rot_cs), es.size, ptr(self.cov), ptr(self.num), ptr(self.den),
             ptr(self.w), ptr(self.intens), s)
        return self.intens


class MStep:
    """MaxLP pattern search of every phaser pixel (a11-a14).

    With ``n_modes`` > 1 the model is ``n_modes`` stacked complex128 images
    and frames carry a reference state ``m*n_ref + s``: each mode is searched
    over the frames assigned to it, with its own ring rescale, in the same
    launches.

    ``screen`` (default): each pattern iteration evaluates every candidate in
    FP32 with a rigorous error bound and only the finalists in FP64; the
    chosen candidates are bit-identical to ``screen=False`` (every candidate
    in FP64).  ``stats`` (device int64[3]) counts the iterations the screen
    settled, the iterations that ran the FP64 pass, and the finalists."""

    def __init__(self, photons, size, num_iter=10, n_modes=1, screen=True):
        self.lib = load()
        self.screen = bool(screen)
        self.ph = photons
        self.device = dev = photons.device
        self.size = int(size)
        self.num_iter = int(num_iter)
        self.n_modes = int(n_modes)
        if self.n_modes < 1:
            raise ValueError('n_modes must be at least 1')
        g = geometry.phaser_pixels(self.size)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype='i4')).to(dev)  # noqa: E731
        self.mask_idx = t(g['mask_idx'])
        self.n_hist_rows = int(g['n_rows'])
        self.ring, self.ring_rows = t(g['ring']), t(g['ring_rows'])
        self.main, self.main_rows = t(g['main']), t(g['main_rows'])
        self.n_ring, self.n_main = int(g['ring'].size), int(g['main'].size)
        self.rescales = torch.empty(self.n_modes * max(1, self.n_ring), dtype=_f64, device=dev)
        self.rescale = torch.empty(self.n_modes, dtype=_f64, device=dev)
        self.fstate = torch.empty(photons.num_data, dtype=_i32, device=dev)
        self.frot = torch.empty(photons.num_data, dtype=_i32, device=dev)
        self.hist = None
        self.nstate = None
        self.stats = torch.zeros(3, dtype=torch.int64, device=dev)
        self.shard = None   # rspi.shard.ShardedMStep when frames are split over ranks

    def _pattern(self, fconv, pixels, rows, n_pix, hist, n_ref, mode, rescale, rescale_out, s):
        if self.screen:
            call('rspi_maxlp_pattern_screened', ptr(fconv), ptr(pixels), ptr(rows), n_pix,
                 ptr(hist), n_ref, ptr(self.nstate), self.n_modes, ptr(self._ref_params),
                 self.size, mode, rescale, self.num_iter, rescale_out, ptr(self.stats), s)
        else:
            call('rspi_maxlp_pattern', ptr(fconv), ptr(pixels), ptr(rows), n_pix, ptr(hist),
                 n_ref, ptr(self.nstate), self.n_modes, ptr(self._ref_params), self.size, mode,
                 rescale, self.num_iter, rescale_out, s)

    def frame_params_from_rmax(self, rmax, num_rot, n_ref):
        """fstate / frot / nstate from the E-step argmax (emc.py:218-224);
        ``n_ref`` (shift, diameter) states per mode, rows
        ``(m*n_ref + s)*num_rot + j``."""
        n_all = int(n_ref) * self.n_modes
        if self.nstate is None or self.nstate.numel() != n_all:
            self.nstate = torch.empty(n_all, dtype=_i32, device=self.device)
        call('rspi_maxlp_frame_params', ptr(rmax), self.ph.num_data, int(num_rot), n_all,
             ptr(self.fstate), ptr(self.frot), ptr(self.nstate), ptr(self.ph.err.t), cur_stream())

    def set_frame_params(self, fstate, frot, nstate):
        self.fstate, self.frot, self.nstate = fstate, frot, nstate

    def pixel_map(self, rot_cs):
        """Per rotation of ``rot_cs`` and detector pixel, the phaser rows whose
        pixel maps onto it (rspi_maxlp_pixel_map), built once per rotation
        table."""
        key = (rot_cs.data_ptr(), tuple(rot_cs.shape))
        if getattr(self, '_pixel_map', None) is not None and self._pixel_map[0] == key:
            return self._pixel_map[1], self._pixel_map[2]
        num_rot, npix, dev = int(rot_cs.shape[0]), self.size * self.size, self.device
        cnt = torch.empty(num_rot * npix, dtype=_i32, device=dev)
        off = torch.empty(num_rot * npix + 1, dtype=_i64, device=dev)
        rows = torch.empty(max(1, num_rot * self.n_hist_rows), dtype=_i32, device=dev)
        call('rspi_maxlp_pixel_map', ptr(rot_cs), num_rot, self.size, ptr(self.mask_idx),
             ptr(cnt), ptr(off), ptr(rows), cur_stream())
        self._pixel_map = (key, off, rows, rot_cs)   # rot_cs kept alive: the key is its address
        return off, rows

    def histogram(self, n_cols, rot_cs):
        """Photons of every phaser pixel per reference state (a11):
        ``n_hist_rows`` x ``n_cols`` int32, from the current frame parameters."""
        need = self.n_hist_rows * n_cols
        if self.hist is None or self.hist.numel() < need:
            self.hist = torch.empty(max(1, need), dtype=_i32, device=self.device)
        hist = self.hist[:max(1, need)]
        hist.zero_()
        ph = self.ph
        num_rot = int(rot_cs.shape[0])
        if num_rot <= PIXEL_MAP_MAX_ROT and num_rot * self.size ** 2 <= PIXEL_MAP_MAX:
            # a table of the rotations' pixel maps, built once per rotation
            # table (the EMC's fixed angles)
            off, rows = self.pixel_map(rot_cs)
            call('rspi_maxlp_histogram_map', ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum),
                 ptr(ph.multi_accum), ptr(ph.place_ones), ptr(ph.place_multi),
                 ptr(ph.count_multi), ph.num_data, ptr(self.fstate), ptr(self.frot), num_rot,
                 self.size, ptr(off), ptr(rows), n_cols, ptr(hist), ptr(ph.err.t), cur_stream())
        else:
            # one rotation per frame (the phaser's own angles): the search per photon
            call('rspi_maxlp_histogram', ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum),
                 ptr(ph.multi_accum), ptr(ph.place_ones), ptr(ph.place_multi),
                 ptr(ph.count_multi), ph.num_data, ptr(self.fstate), ptr(self.frot), ptr(rot_cs),
                 self.size, ptr(self.mask_idx), self.n_hist_rows, n_cols, ptr(hist),
                 ptr(ph.err.t), cur_stream())
        if self.shard is not None:
            # sums over every rank's frames: the histogram of the whole dataset
            self.shard.reduce_histogram(hist, self.nstate)
        return hist

    def grid(self, fconv, ref_params, rot_cs, scales, n_phase=64, n_amp=32):
        """Polar grid search of the per-pixel NLL over the main phaser pixels
        (one mode): ``fconv`` updated in place; returns the per-pixel NLL
        values of the chosen points (without the F-independent term)."""
        if self.n_modes != 1:
            raise ValueError('the grid search takes one mode')
        if self.shard is not None:
            raise ValueError('the grid search runs on one GPU (its per-state scale sums are '
                             'frame-local)')
        n_ref = int(ref_params.shape[0])
        hist = self.histogram(n_ref, rot_cs)
        ssum = torch.empty(n_ref, dtype=_f64, device=self.device)
        best = torch.empty(max(1, self.n_main), dtype=_f64, device=self.device)
        call('rspi_maxlp_grid', ptr(fconv), ptr(self.main), ptr(self.main_rows), self.n_main,
             ptr(hist), n_ref, ptr(self.fstate), ptr(scales), self.ph.num_data, ptr(ref_params),
             self.size, int(n_phase), int(n_amp), ptr(ssum), ptr(best), ptr(self.ph.err.t),
             cur_stream())
        return best[:self.n_main]

    def run(self, fconv, ref_params, rot_cs, main=True):
        """Update ``fconv`` (complex128 device tensor, ``n_modes`` x P) in place:
        the ring pass and the global rescale, then (``main``) the main pass."""
        n_ref = int(ref_params.shape[0])
        nm = self.n_modes
        if fconv.numel() != nm * self.size ** 2:
            raise ValueError('fconv must hold %d model(s) of %d pixels' % (nm, self.size ** 2))
        if self.nstate is None or self.nstate.numel() != nm * n_ref:
            raise ValueError('frame parameters are not set for %d x %d states' % (nm, n_ref))
        hist = self.histogram(n_ref * nm, rot_cs)
        s = cur_stream()
        ph = self.ph
        self._ref_params = ref_params
        self._pattern(fconv, self.ring, self.ring_rows, self.n_ring, hist, n_ref, 0, None,
                      ptr(self.rescales), s)
        if self.n_ring > 0:
            for m in range(nm):
                call('rspi_mean', ptr(self.rescales[m * self.n_ring:]), self.n_ring,
                     ptr(self.rescale[m:]), s)
        else:
            self.rescale.fill_(float('nan'))   # np.mean of an empty ring
        if main and self.shard is None:
            self._pattern(fconv, self.main, self.main_rows, self.n_main, hist, n_ref, 1,
                          ptr(self.rescale), None, s)
        elif main:
            # this rank's block of the main pixels, then every rank's updates
            lo, hi = self.shard.main_block()
            self._pattern(fconv, self.main[lo:], self.main_rows[lo:], hi - lo, hist, n_ref, 1,
                          ptr(self.rescale), None, s)
            self.shard.gather_main(fconv, self.main[lo:hi])
        return fconv
