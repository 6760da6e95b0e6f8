"""MaxLP phaser on the GPU -- drop-in for the reference ``maxLP.py``.

``MaxLPhaser(data_fname, size=185, num_data=-1)`` keeps the reference's
constructor and ``_run_phaser(model, sx_vals, sy_vals, dia_vals, ang_vals)``
(maxLP.py:304-340), with the same q grids, masks and candidate pattern
(``qx``, ``qy``, ``qrad``, ``mask``, ``rmask``, ``pattern``), the
``photons`` CSR matrix and the per-pixel methods (``get_photons_pixel``,
``get_fref_d``, ``get_pixel_constants``, ``get_rescale_pixel``,
``get_logq_pixel``, ``iterate_pixel_pattern``, ``run_pixel_pattern``,
``_get_sphere``, ``get_fcalc_all``), all on the device.  The per-pixel
pattern search runs in librspi (one CTA per pixel, all 1089 candidates at
once); see csrc/maxlp.cu for the exact sparse/analytic rewrite of
``get_logq_pixel``.
"""
import os
import sys
import warnings

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from rspi import geometry  # noqa: E402
from rspi.device import MStep, cur_stream, ptr  # noqa: E402
from rspi import lib as rlib  # noqa: E402
from rspi.lib import call  # noqa: E402


class MaxLPhaser():
    '''Reconstruction of object from holographic data using maximum likelihood and pattern search'''
    def __init__(self, data_fname, size=185, num_data=-1, dataset=None, device=None,
                 num_iter=10, num_modes=1, screen=True):
        self.size = size
        self.num_iter = num_iter
        self.num_modes = int(num_modes)
        if dataset is None:
            from dset import Dataset
            dataset = Dataset(data_fname, size ** 2, device=device, num_data=num_data)
        elif 0 <= num_data < dataset.num_data:
            raise ValueError('num_data < dataset.num_data needs the phaser to read its own file')
        self.dset = dataset
        self.num_data = dataset.num_data
        self.device = dataset.device
        self.qx, self.qy, self.qrad, self.mask, self.rmask = geometry.phaser_qvals(size)
        self.mask_ind = np.where(self.mask.ravel())[0]
        self._gen_pattern(8)
        self.counts = dataset.photons.counts
        self.mean_count = dataset.photons.mean_count
        self.mstep = MStep(dataset.photons, size, num_iter, n_modes=self.num_modes,
                           screen=screen)
        # model-refinement masks (maxLP.py:28-33): integer-centred radius, the
        # pixels the Fourier projection takes from the data, the support
        mx, my = np.indices((size,) * 2, dtype='f8')
        self.mx_ind = torch.from_numpy(mx.ravel() - size // 2).to(self.device)
        self.my_ind = torch.from_numpy(my.ravel() - size // 2).to(self.device)
        self.mrad = torch.sqrt(self.mx_ind ** 2 + self.my_ind ** 2)
        self.minvsuppmask = torch.ones((size,) * 2, dtype=torch.bool, device=self.device)
        self.minvmask = self._get_invmask(4)
        self.badpixmask = torch.ones(size ** 2, dtype=torch.bool, device=self.device)
        self._phase_work = None

    def _gen_pattern(self, nmax):
        '''33x33 candidate offsets (maxLP.py:45-48)'''
        ind = np.arange(-nmax, nmax + 0.5, 0.5)
        x, y = np.meshgrid(ind, ind, indexing='ij')
        self.pattern = (x + 1j * y).ravel()

    def _get_rot(self, ang):
        '''Rotation matrices (maxLP.py:255-258)'''
        c = np.cos(ang)
        s = np.sin(ang)
        return np.array([[c, -s], [s, c]])

    # -- per-pixel, per-frame API (maxLP.py:107-114, 154-253) ------------
    # The reference's own search walks one pixel at a time over every frame;
    # these run it through librspi on the frames' parameters of the last
    # _run_phaser call, returning CUDA tensors as the reference returns CuPy
    # arrays.

    @property
    def photons(self):
        '''Photon counts as a sparse CSR matrix, frames x pixels
        (maxLP.py:50-71), on the device.'''
        if getattr(self, '_photons_csr', None) is None:
            ph = self.dset.photons
            n = self.num_data
            rows_o = torch.repeat_interleave(torch.arange(n, device=self.device), ph.ones.long())
            rows_m = torch.repeat_interleave(torch.arange(n, device=self.device), ph.multi.long())
            idx = torch.stack([torch.cat([rows_o, rows_m]),
                               torch.cat([ph.place_ones.long(), ph.place_multi.long()])])
            val = torch.cat([torch.ones(rows_o.numel(), dtype=torch.float64, device=self.device),
                             ph.count_multi.double()])
            with warnings.catch_warnings():   # torch's notes on sparse tensors
                warnings.simplefilter('ignore', UserWarning)
                coo = torch.sparse_coo_tensor(idx, val, (n, self.size ** 2),
                                              check_invariants=True).coalesce()
                self._photons_csr = coo.to_sparse_csr()
        return self._photons_csr

    def _frame_tables(self):
        '''Per-frame (cos, sin) of -angle and (shift x, shift y, diameter) of
        the last _run_phaser call, on the device.'''
        if getattr(self, 'ang', None) is None:
            raise ValueError('the per-frame parameters are set by _run_phaser')
        if getattr(self, '_ftab', None) is None:
            rot = torch.from_numpy(geometry.phaser_rotation_table(self.ang)).to(self.device)
            fp = np.ascontiguousarray(np.stack([self.shifts[:, 0], self.shifts[:, 1],
                                                self.diams], axis=1), dtype='f8')
            self._ftab = (rot, torch.from_numpy(fp).to(self.device))
        return self._ftab

    def _pixel_frames(self, d_vals, t):
        rot, fp = self._frame_tables()
        ph = self.dset.photons
        if d_vals is None:
            dv, n = None, self.num_data
        else:
            dv = torch.as_tensor(np.ascontiguousarray(np.asarray(d_vals).ravel(), dtype='i4'))
            dv = dv.to(self.device)
            n = dv.numel()
        k = torch.empty(n, dtype=torch.float64, device=self.device)
        fref = torch.empty(n, dtype=torch.complex128, device=self.device)
        call('rspi_maxlp_pixel_frames', int(t), self.size, ptr(dv), n, ptr(ph.ones),
             ptr(ph.multi), ptr(ph.ones_accum), ptr(ph.multi_accum), ptr(ph.place_ones),
             ptr(ph.place_multi), ptr(ph.count_multi), ph.num_data, ptr(rot), ptr(fp), ptr(k),
             ptr(fref), ptr(ph.err.t), cur_stream())
        ph.err.check('MaxLP pixel frames')
        return k, fref

    def get_photons_pixel(self, d_vals, t):
        '''Photons of frames d_vals at model pixel t (maxLP.py:245-253)'''
        return self._pixel_frames(d_vals, t)[0]

    def get_fref_d(self, d_vals, t):
        '''Reference amplitude of frames d_vals at model pixel t (maxLP.py:238-243)'''
        return self._pixel_frames(d_vals, t)[1]

    def get_pixel_constants(self, t, frac=None):
        '''k_d and fref_d of every frame (or a random fraction) at pixel t
        (maxLP.py:107-114)'''
        d_vals = None
        if frac is not None:
            d_vals = np.random.choice(self.num_data, int(np.round(self.num_data * frac)),
                                      replace=False)
        k, fref = self._pixel_frames(d_vals, t)
        return {'k_d': k, 'fref_d': fref}

    def _candidates(self, fobj_t):
        if isinstance(fobj_t, torch.Tensor):
            c = fobj_t.to(self.device, torch.complex128).reshape(-1).contiguous()
        else:
            c = torch.from_numpy(np.ascontiguousarray(np.atleast_1d(np.asarray(
                fobj_t, dtype=np.complex128)).ravel())).to(self.device)
        return c

    def _pixel_values(self, cands, const, mode, rescale):
        n = int(const['k_d'].numel())
        out = torch.empty(cands.numel(), dtype=torch.float64, device=self.device)
        rvec, rs = None, 0.
        if isinstance(rescale, torch.Tensor) or (rescale is not None and np.ndim(rescale) > 0):
            rvec = torch.as_tensor(rescale, dtype=torch.float64).to(self.device)
            rvec = rvec.reshape(-1).contiguous()
            if rvec.numel() != cands.numel():
                rvec = rvec.expand(cands.numel()).contiguous()
        elif rescale is not None:
            rs = float(rescale)
        # operands held in locals: a temporary passed straight to ptr() is
        # freed before the launch and its block may be handed to the next one
        k_d, fref_d = const['k_d'].contiguous(), const['fref_d'].contiguous()
        call('rspi_maxlp_pixel_values', ptr(cands), cands.numel(), ptr(k_d), ptr(fref_d), n,
             mode, rs, ptr(rvec), ptr(out), cur_stream())
        return out

    def get_rescale_pixel(self, fobj_t, t, const=None):
        '''mean_d k_d / mean_d |f + fref_d|^2 per candidate f (maxLP.py:216-228)'''
        if const is None:
            const = self.get_pixel_constants(t)
        return self._pixel_values(self._candidates(fobj_t), const, 0, None)

    def get_logq_pixel(self, fobj_t, t, rescale=None, const=None):
        '''Log-likelihood of candidates f at model pixel t (maxLP.py:181-197)'''
        if const is None:
            const = self.get_pixel_constants(t)
        cands = self._candidates(fobj_t)
        if rescale is None:
            rescale = self._pixel_values(cands, const, 0, None)
        return self._pixel_values(cands, const, 1, rescale)

    def _argmax(self, vals):
        '''First index of the maximum (a NaN counts as the maximum), on the device.'''
        v = vals.reshape(-1, 1).contiguous()
        mx = torch.empty(1, dtype=torch.float64, device=self.device)
        im = torch.empty(1, dtype=torch.int32, device=self.device)
        call('rspi_frame_reduce', ptr(v), 1, v.shape[0], 1, ptr(mx), ptr(im), None, cur_stream())
        return int(im.item())

    def iterate_pixel_pattern(self, fobj_t, t, step, rescale=None, const=None):
        '''One pattern-search step at pixel t (maxLP.py:169-179)'''
        if const is None:
            const = self.get_pixel_constants(t)
        fobj_t = complex(fobj_t)
        vals = self.get_logq_pixel(fobj_t + self.pattern * step, t, rescale=rescale,
                                   const=const)
        imax = self._argmax(vals)
        retf = fobj_t + self.pattern[imax] * step
        if imax == self.pattern.size // 2:   # centre of the pattern
            return retf, step / (self.pattern.size ** 0.5 / 5)
        return retf, step

    def run_pixel_pattern(self, fobj, t, num_iter=10, rescale=None, frac=None):
        '''Pattern search of model pixel t over every frame (maxLP.py:154-167)'''
        if isinstance(fobj, torch.Tensor):
            fobj_t = complex(fobj.reshape(-1)[t].item())
        else:
            fobj_t = complex(np.asarray(fobj).ravel()[t])
        const = self.get_pixel_constants(t, frac=frac)
        step = abs(fobj_t) / 4.
        for _ in range(num_iter):
            fobj_t_new, step_new = self.iterate_pixel_pattern(fobj_t, t, step, rescale, const)
            with np.errstate(divide='ignore', invalid='ignore'):
                if np.float64(step_new) / np.float64(abs(fobj_t_new)) < 1.e-3:
                    break
            fobj_t = fobj_t_new
            step = step_new
        return fobj_t

    def _get_sphere(self, dia):
        '''Sphere transform for a diameter (maxLP.py:266-269), on the device'''
        out = torch.empty((self.size, self.size), dtype=torch.float64, device=self.device)
        call('rspi_maxlp_fcalc', self.size, float(dia), 0., 0., None, ptr(out), None,
             cur_stream())
        return out

    def get_fcalc_all(self, fobj, dia, shift):
        '''Holographic combination of model and spherical reference
        (maxLP.py:260-264), on the device'''
        f = self._candidates(fobj)
        if f.numel() != self.size ** 2:
            raise ValueError('fobj must hold %d pixels' % self.size ** 2)
        out = torch.empty((self.size, self.size), dtype=torch.complex128, device=self.device)
        call('rspi_maxlp_fcalc', self.size, float(dia), float(shift[0]), float(shift[1]),
             ptr(f), None, ptr(out), cur_stream())
        return out

    def _run_phaser(self, model, sx_vals, sy_vals, dia_vals, ang_vals, modes=None):
        '''Ring pass, global rescale and main pass over every phaser pixel
        (maxLP.py:304-340).  Frames may carry any (shift, diameter, angle);
        frames sharing a (shift, diameter) share the reference amplitude.
        With ``num_modes`` > 1, ``model`` is (num_modes, P) and ``modes[d]``
        names the model frame d belongs to; each mode is searched over its
        own frames.'''
        nm = self.num_modes
        if modes is None:
            if nm > 1:
                raise ValueError('modes (one per frame) are required with num_modes > 1')
            modes = np.zeros(self.num_data, dtype='i4')
        modes = np.asarray(modes).ravel()
        if modes.size != self.num_data or modes.min() < 0 or modes.max() >= nm:
            raise ValueError('modes must give each frame a mode in [0, %d)' % nm)
        sx = np.asarray(sx_vals, dtype='f8').ravel()
        sy = np.asarray(sy_vals, dtype='f8').ravel()
        dia = np.asarray(dia_vals, dtype='f8').ravel()
        ang = np.asarray(ang_vals, dtype='f8').ravel()
        if not (sx.size == sy.size == dia.size == ang.size == self.num_data):
            raise ValueError('one shift/diameter/angle per frame is required')
        self.shifts = np.array([sx, sy]).T
        self.diams = dia
        self.ang = ang
        self._ftab = None   # the per-pixel API's frame tables follow these
        triples = np.stack([sx, sy, dia], axis=1)
        ref, fstate = np.unique(triples, axis=0, return_inverse=True)
        dev = self.device
        ref_params = torch.from_numpy(np.ascontiguousarray(ref)).to(dev)
        fstate = modes.astype(np.int64) * ref.shape[0] + fstate.ravel()
        fstate_t = torch.from_numpy(fstate.astype('i4')).to(dev)
        frot_t = torch.arange(self.num_data, dtype=torch.int32, device=dev)
        nstate = torch.from_numpy(np.bincount(fstate, minlength=nm * ref.shape[0]).astype('i4')).to(dev)
        rot_cs = torch.from_numpy(geometry.phaser_rotation_table(ang)).to(dev)
        self.mstep.set_frame_params(fstate_t, frot_t, nstate)
        model = np.array(model, dtype=np.complex128)
        fconv = torch.from_numpy(model.ravel()).to(dev)
        self.mstep.run(fconv, ref_params, rot_cs)
        out = fconv.cpu().numpy().reshape(model.shape)
        self.dset.photons.err.check('MaxLP phaser')
        return out

    # -- model refinement: error reduction and difference map --------------
    # (maxLP.py:271-298, 342-354) through librspi's centred transforms; the
    # images are flat complex128 CUDA tensors of size**2 pixels.

    def _get_invmask(self, r):
        '''Pixels taken from the data by the Fourier projection: r <= mrad <
        size//2 (maxLP.py:71-75)'''
        self.minvmask = (self.mrad >= r) & (self.mrad < self.size // 2)
        return self.minvmask

    def _image(self, x):
        t = torch.as_tensor(np.asarray(x) if not torch.is_tensor(x) else x)
        t = t.to(self.device, torch.complex128).reshape(-1).contiguous()
        if t.numel() != self.size ** 2:
            raise ValueError('an image of %d pixels is required' % self.size ** 2)
        return t

    @staticmethod
    def _bytes(mask):
        return mask.reshape(-1).to(torch.uint8).contiguous()

    def _work(self):
        if self._phase_work is None:
            self._phase_work = torch.empty(8 * self.size ** 2, dtype=torch.float64,
                                           device=self.device)
        return self._phase_work

    def proj_fourier(self, fconv, x):
        '''x with the data pixels (minvmask) replaced by fconv\'s
        (maxLP.py:271-274)'''
        fconv, x = self._image(fconv), self._image(x)
        out = torch.empty_like(x)
        inv = self._bytes(self.minvmask)
        call('rspi_phase_proj_fourier', ptr(fconv), ptr(inv), ptr(x), ptr(out), self.size,
             cur_stream())
        return out

    def proj_real(self, x):
        '''Real-space projection (maxLP.py:276-280): real part of the centred
        inverse transform, negatives and pixels outside the support set to 0,
        transformed back'''
        x = self._image(x)
        out = torch.empty_like(x)
        supp = self._bytes(self.minvsuppmask)
        call('rspi_phase_proj_real', ptr(x), ptr(supp), ptr(out), ptr(self._work()), self.size,
             cur_stream())
        return out

    def _refine(self, fconv, x, n_dm, n_er):
        fconv = self._image(fconv)
        out = self._image(x).clone()
        # both masks held until the launch: a temporary handed straight to
        # ptr() goes back to the allocator at once, and the second mask's copy
        # could then land in the first one's block before the kernel reads it
        inv, supp = self._bytes(self.minvmask), self._bytes(self.minvsuppmask)
        call('rspi_phase_refine', ptr(fconv), ptr(inv), ptr(supp), ptr(out), ptr(self._work()),
             self.size, int(n_dm), int(n_er), cur_stream())
        rlib.launch_count += 5 * (int(n_dm) + int(n_er))
        return out

    def er(self, fconv, x):
        '''One error-reduction step (maxLP.py:282-284)'''
        return self._refine(fconv, x, 0, 1)

    def diffmap(self, fconv, x):
        '''One difference-map step (maxLP.py:286-289)'''
        return self._refine(fconv, x, 1, 0)

    def _get_support(self, fconv):
        '''True outside the support (maxLP.py:292-298): fconv tapered by
        expit((mrad - 12) / 2), centred inverse transform, |real part|
        smoothed by a sigma-3 Gaussian, not above 1.2e-4'''
        fconv = self._image(fconv)
        supp = torch.empty(self.size ** 2, dtype=torch.uint8, device=self.device)
        call('rspi_phase_support', ptr(fconv), self.size, 12., 0.5, 3., 12, 1.2e-4, ptr(supp),
             ptr(self._work()), cur_stream())
        return supp.bool().reshape((self.size,) * 2)

    def _get_tot_mask(self, fconv):
        '''Data mask without the pixels whose real part is at or below -0.2
        (maxLP.py:299-302)'''
        self.badpixmask = self._image(fconv).real > -0.2
        return self.badpixmask & self.minvmask

    def _improve_model(self, fconv, update_masks=True):
        '''Support from fconv (with update_masks), then 10 difference-map and
        5 error-reduction iterations starting from fconv (maxLP.py:342-354);
        a complex128 CUDA tensor of size**2 pixels'''
        print('Starting diffmap and er')
        fconv = self._image(fconv)
        if update_masks is True:
            self.minvsuppmask = self._get_support(fconv)
        out = self._refine(fconv, fconv, 10, 5)
        print('Done...')
        return out

    def run_from_rmax(self, fconv, rmax, num_rot, state_values, rot_cs):
        '''Device path used by EMC: frames' parameters come straight from the
        E-step argmax (emc.py:218-224) without leaving the GPU.  ``fconv`` is
        a complex128 device tensor updated in place.'''
        self.mstep.frame_params_from_rmax(rmax, num_rot, state_values.shape[0])
        return self.mstep.run(fconv, state_values, rot_cs)
