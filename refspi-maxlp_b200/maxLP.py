"""MaxLP phaser on the GPU -- drop-in for the reference ``maxLP.py``.

``MaxLPhaser(data_fname, size=185, num_data=-1)`` keeps the reference's
constructor and ``_run_phaser(model, sx_vals, sy_vals, dia_vals, ang_vals)``
(maxLP.py:304-340), with the same q grids, masks and candidate pattern
(``qx``, ``qy``, ``qrad``, ``mask``, ``rmask``, ``pattern``).  The per-pixel
pattern search runs in librspi (one CTA per pixel, all 1089 candidates at
once); see csrc/maxlp.cu for the exact sparse/analytic rewrite of
``get_logq_pixel``.
"""
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from rspi import geometry  # noqa: E402
from rspi.device import MStep  # noqa: E402


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

    def get_fref_d(self, d_vals, t):
        '''Reference amplitude of frames d_vals at model pixel t (maxLP.py:238-243)'''
        sval = np.pi * self.qrad[t] * self.diams[d_vals]
        fref = (np.sin(sval) - sval * np.cos(sval)) / sval ** 3
        ramp = np.exp(1j * 2 * np.pi * (self.qx[t] * self.shifts[d_vals, 0] +
                                        self.qy[t] * self.shifts[d_vals, 1]))
        return fref * ramp

    def get_fcalc_all(self, fobj, dia, shift):
        '''Holographic combination of model and spherical reference (maxLP.py:260-264)'''
        qx2d = self.qx.reshape((self.size,) * 2)
        qy2d = self.qy.reshape((self.size,) * 2)
        return fobj + self._get_sphere(dia) * np.exp(1j * 2 * np.pi * (qx2d * shift[0] + qy2d * shift[1]))

    def _get_sphere(self, dia):
        '''Sphere transform for a diameter (maxLP.py:266-269)'''
        sval = np.pi * self.qrad.reshape((self.size,) * 2) * dia
        return (np.sin(sval) - sval * np.cos(sval)) / sval ** 3

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

    def run_from_rmax(self, fconv, rmax, num_rot, state_values, rot_cs):
        '''Device path used by EMC: frames' parameters come straight from the
        E-step argmax (emc.py:218-224) without leaving the GPU.  ``fconv`` is
        a complex128 device tensor updated in place.'''
        self.mstep.frame_params_from_rmax(rmax, num_rot, state_values.shape[0])
        return self.mstep.run(fconv, state_values, rot_cs)
