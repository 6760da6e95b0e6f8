#!/usr/bin/env python
'''Generator of objects (homo- and heterogeneous) and their holographic
diffraction frames: the reference's make_data.py (DataGenerator, the
``[make_data]`` / ``[parameters]`` configuration keys and the CLI), with the
per-frame loop (make_data.py:289-329) replaced by batched librspi kernels
(csrc/simulate.cu): frame model, holographic intensity, mask, normalisation,
rotation, background, Poisson counts and the sparse photon lists for
thousands of frames per launch.

Differences from the reference, all of them additions:
* ``[make_data] seed`` (optional): seeds every draw (object discs, frame
  parameters, photon counts), so a configuration reproduces its file; the
  reference draws from unseeded generators.  Photon counts come from a
  counter-based generator keyed by (seed, frame, pixel).
* ``[make_data] frames_per_batch`` (optional): frames per launch (default: as
  many as fit in an eighth of the free device memory, at most 4,096).
* The output file is HDF5 (``.h5``, written by rspi.h5lite: h5py is not
  required) or ``.npz`` in the photons-file layout; datasets already in the
  file that this run does not write are kept, as with h5py's append mode.
* The deterministic object (``create_random = no``) raises ValueError where
  the reference's placement loop would not terminate (a disc leaving the
  detector), and ``homo`` / ``mix`` / ``blur`` without ``object_hetro``
  raise ValueError where the reference fails on an undefined name.
'''
import argparse
import configparser
import os
import os.path as op
import sys
import time

import numpy as np
import torch

sys.path.insert(0, op.dirname(op.abspath(__file__)))
from rspi import photonfile  # noqa: E402
from rspi.device import ErrorWord, cur_stream, ptr  # noqa: E402
from rspi.lib import call, load  # noqa: E402

_f64 = torch.float64
KINDS = {'iso': 0, 'homo': 1, 'mix': 2, 'blur': 3}


class DataGenerator():
    def __init__(self, config_file, device=None):
        config = configparser.ConfigParser()
        config.read(config_file)

        self.num_data = config.getint('make_data', 'num_data')
        self.fluence = config.get('make_data', 'fluence', fallback='constant')
        self.mean_count = config.getfloat('make_data', 'mean_count')

        self.dia_params = [float(s) for s in config.get('make_data', 'dia_params').split()]
        self.shift_sigma = config.getfloat('make_data', 'shift_sigma')
        self.wobble_sigma = config.getfloat('make_data', 'wobble_sigma')

        s = [int(_) for _ in config.get('parameters', 'size').split()]
        use_padding = config.getboolean('make_data', 'use_zero_padding', fallback=False)
        self.size = s[1] if use_padding else s[0]

        self.object_hetro = config.getboolean('make_data', 'object_hetro', fallback=False)
        object_type = config.get('make_data', 'object_type', fallback='mix')
        if object_type not in KINDS:
            raise ValueError('Object type needs to be from (iso, homo, mix or blur')
        self.object_type = object_type
        self.gen_iso = object_type == 'iso'
        self.gen_homo = object_type == 'homo'
        self.gen_mix = object_type == 'mix'
        self.gen_blur = object_type == 'blur'

        self.create_random = config.getboolean('make_data', 'create_random', fallback=False)
        self.bg_count = config.getfloat('make_data', 'bg_count', fallback=None)
        self.rel_scale = config.getfloat('make_data', 'rel_scale')

        cdir = op.dirname(config_file)
        self.output_folder = op.join(cdir, config.get('make_data', 'output_folder'))
        self.out_photons_file = os.path.join(cdir, config.get('make_data', 'out_photons_file'))

        if self.fluence not in ['constant', 'gamma']:
            raise ValueError('make_data:fluence needs to be either constant (default) or gamma')

        seed = config.get('make_data', 'seed', fallback='').strip()
        self.seed = int(seed) if seed else None
        self.rng = np.random.default_rng(self.seed)
        self.frames_per_batch = config.getint('make_data', 'frames_per_batch', fallback=0)

        self.lib = load()
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.err = ErrorWord(self.device)
        z = lambda: torch.zeros((self.size, self.size), dtype=_f64, device=self.device)  # noqa
        self.object = z()
        self.object_sum = 0
        if self.object_hetro:
            self.wobble_object = z()
            self.wobble_object_sum = 0
        self.bgmask = z()
        self.bgmask_sum = 0

    # -- objects -----------------------------------------------------------

    def _add_disc(self, acc, c0, c1, rad):
        '''acc += 1 - (r / rad)^2 where r <= rad (make_data.py:104-105)'''
        x, y = self._xy
        r = torch.sqrt((x - c0) ** 2 + (y - c1) ** 2)
        inside = r <= rad
        acc[inside] += 1. - (r[inside] / rad) ** 2

    def _discs(self, acc, n, random, rad_det, cen_det, rad_rand, cen_rand, what):
        mcen = self.size // 2
        for i in range(n):
            if random:
                rad = rad_rand(self.rng.random())
                while True:
                    c0, c1 = cen_rand(self.rng.random(2))
                    if float(np.sqrt((c0 - mcen) ** 2 + (c1 - mcen) ** 2) + rad) < mcen:
                        break
            else:
                rad = rad_det(i)
                c0, c1 = cen_det(i)
                if not float(np.sqrt((c0 - mcen) ** 2 + (c1 - mcen) ** 2) + rad) < mcen:
                    raise ValueError('%s disc %d of the default object leaves a %d-pixel '
                                     'detector' % (what, i, self.size))
            self._add_disc(acc, float(c0), float(c1), float(rad))

    def make_obj(self, bg=False):
        '''Object (or, with bg, background) of parabolic discs
        (make_data.py:95-167): 55 discs, and 25 wobble discs for a
        heterogeneous object; random with create_random, else at fixed
        positions.  The object goes to the output file as ``solution`` (or
        ``rigid`` and ``wobble``).'''
        size = self.size
        mask = self.bgmask if bg else self.object
        mcen = size // 2
        self._xy = [t.to(self.device) for t in torch.meshgrid(
            torch.arange(size, dtype=_f64), torch.arange(size, dtype=_f64), indexing='ij')]
        self._discs(
            mask, 55, self.create_random,
            lambda i: (0.7 + 0.3 * (np.cos(2.5 * i) - np.sin(i / 4))) * size / 20.,
            lambda i: ((3 * np.sin(2 * i) + 0.5 * np.sin(i / 2)) * size / 45. + mcen * 4. / 4.4,
                       (0.5 * np.cos(i / 2) + 3 * np.cos(i / 2)) * size / 45. + mcen * 4. / 4.4),
            lambda u: (0.7 + 0.3 * u) * size / 25.,
            lambda u: (u[0] * size / 5. + mcen * 4. / 5., u[1] * size / 5. + mcen * 4. / 5.),
            'object')
        if self.object_hetro:
            wobble_mask = self.bgmask if bg else self.wobble_object
            self._discs(
                wobble_mask, 25, self.create_random,
                lambda i: (0.7 + 0.3 * (np.sin(i) - np.cos(i / 2))) * size / 30.,
                lambda i: ((np.sin(2 * i) - 3 * np.cos(i)) * size / 60. + mcen * 4.6 / 7.,
                           (np.cos(i) - np.sin(i / 2)) * size / 60. + mcen * 4.6 / 7.),
                lambda u: (0.7 + 0.3 * u) * size / 22.,
                lambda u: (u[0] * size / 10. + mcen * 4. / 6., u[1] * size / 10. + mcen * 4. / 6.),
                'wobble')
        total = float(mask.sum()) + (float(wobble_mask.sum()) if self.object_hetro else 0.)
        if bg:
            self.bgmask_sum = total
            return
        self.object_sum = total
        if self.object_hetro:
            self.wobble_object = wobble_mask
            photonfile.update_datasets(self.out_photons_file,
                                       {'rigid': mask.cpu().numpy(),
                                        'wobble': wobble_mask.cpu().numpy()})
        else:
            photonfile.update_datasets(self.out_photons_file, {'solution': mask.cpu().numpy()})

    def parse_obj(self, bg=False):
        '''Object (or background, scaled to bg_count photons) from the output
        file's ``solution`` / ``wobble`` (or ``bg``) datasets
        (make_data.py:169-196).'''
        dset_name = 'bg' if bg else 'solution'
        wobble_dset_name = 'bg' if bg else 'wobble'
        f = photonfile.PhotonsFile(self.out_photons_file)
        mask = torch.as_tensor(np.array(f[dset_name], dtype='f8')).to(self.device)
        if self.object_hetro:
            wobble_mask = torch.as_tensor(np.array(f[wobble_dset_name], dtype='f8')) \
                .to(self.device)
        if bg:
            mask *= self.bg_count / mask.sum()
            self.bgmask_sum = float(mask.sum())
            self.bgmask = mask
            if self.object_hetro:
                wobble_mask *= self.bg_count / wobble_mask.sum()
                self.bgmask_sum = float(mask.sum() + wobble_mask.sum())
                self.bgmask = mask + wobble_mask
        else:
            self.object_sum = float(mask.sum())
            self.object = mask
            if self.object_hetro:
                self.object_sum = float(mask.sum() + wobble_mask.sum())
                self.wobble_object = wobble_mask

    # -- frames ------------------------------------------------------------

    def _centred_fft(self, obj):
        '''fftshift(fftn(ifftshift(obj))) (make_data.py:282-284) by
        librspi's centred transform'''
        size = self.size
        x = obj.to(torch.complex128).reshape(-1).contiguous()
        out = torch.empty_like(x)
        work = torch.empty_like(x)
        call('rspi_cdft2', ptr(x), ptr(out), ptr(work), size, 0, cur_stream())
        return out

    def _batch(self):
        if self.frames_per_batch > 0:
            return min(self.frames_per_batch, 65535)
        free, _ = torch.cuda.mem_get_info(self.device)
        per_frame = self.size ** 2 * 12
        return int(max(1, min(4096, free // 8 // per_frame)))

    def make_data(self, parse=False):
        '''Frames of the object (make_data.py:199-333): per frame a fluence
        scale (constant, or gamma(2, 0.5)), a sphere shift N(0,
        shift_sigma^2) per axis, a diameter N(dia_params[0],
        dia_params[1]^2), an angle U(0, 2 pi) and, for a heterogeneous
        object, a wobble N(0, wobble_sigma^2); the photon counts are Poisson
        draws of the rotated, normalised holographic intensity.'''
        if self.object_sum == 0.:
            if parse:
                self.parse_obj()
            else:
                self.make_obj()
        if self.bg_count is not None:
            if parse:
                self.parse_obj(bg=True)
            else:
                self.make_obj(bg=True)
        if not self.gen_iso and not self.object_hetro:
            raise ValueError('object_type %s needs object_hetro = yes' % self.object_type)

        n, size, rng = self.num_data, self.size, self.rng
        out = {}
        if self.bgmask_sum > 0:
            out['bg'] = self.bgmask.cpu().numpy()
        out['num_pix'] = np.array([size ** 2])
        scale = rng.gamma(2., 0.5, n) if self.fluence == 'gamma' else np.ones(n, dtype='f8')
        out['scale'] = scale
        shifts = rng.standard_normal((n, 2)) * self.shift_sigma
        out['true_shifts'] = shifts
        if self.object_hetro:
            wobbles = rng.standard_normal((n, 2)) * self.wobble_sigma
            out['true_wobbles'] = wobbles.copy()
        diameters = rng.standard_normal(n) * self.dia_params[1] + self.dia_params[0]
        out['true_diameters'] = diameters
        angles = rng.random(n) * 2. * np.pi
        out['true_angles'] = angles
        # the wobble amplitude each frame uses (make_data.py:296,300: 4.5 for
        # homo and mix; the file keeps the drawn values)
        if self.gen_homo or self.gen_mix:
            w_used = np.full(n, 4.5)
        elif self.gen_blur:
            w_used = wobbles[:, 0].copy()
        else:
            w_used = np.zeros(n)
        seed = int(rng.integers(0, 2 ** 63))

        dev = self.device
        model = self._centred_fft(self.object)
        wob = self._centred_fft(self.wobble_object) if self.object_hetro else None
        bg = self.bgmask.reshape(-1).contiguous() if self.bg_count is not None else None
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype='f8')).to(dev)  # noqa
        shifts_d, dia_d, scale_d, w_d = t(shifts.ravel()), t(diameters), t(scale), t(w_used)
        cs_d = t(np.stack([np.cos(angles), np.sin(angles)], 1).ravel())
        kind = KINDS[self.object_type]
        mask_value = 2. if self.object_hetro else 1.
        npix = size ** 2
        batch = self._batch()
        view = torch.empty((batch, npix), dtype=_f64, device=dev)
        counts = torch.empty((batch, npix), dtype=torch.int32, device=dev)
        n1 = torch.empty(batch, dtype=torch.int32, device=dev)
        nm = torch.empty(batch, dtype=torch.int32, device=dev)
        off1 = torch.empty(batch + 1, dtype=torch.int64, device=dev)
        offm = torch.empty(batch + 1, dtype=torch.int64, device=dev)
        lists = {k: [] for k in ('ones', 'multi', 'place_ones', 'place_multi', 'count_multi')}
        s = cur_stream()
        stime = time.time()
        photons = 0
        for f0 in range(0, n, batch):
            b = min(batch, n - f0)
            call('rspi_sim_views', ptr(model), ptr(wob), kind, f0, b, ptr(w_d[f0:]),
                 ptr(shifts_d[2 * f0:]), ptr(dia_d[f0:]), ptr(scale_d[f0:]), self.rel_scale,
                 self.mean_count, mask_value, size, ptr(view), ptr(self.err.t), s)
            call('rspi_sim_counts', ptr(view), f0, b, ptr(cs_d[2 * f0:]), ptr(bg), size, seed,
                 ptr(counts), None, ptr(self.err.t), s)
            call('rspi_sim_sparse_counts', ptr(counts), b, npix, ptr(n1), ptr(nm), s)
            call('rspi_scan_rows', ptr(n1), b, ptr(off1), s)
            call('rspi_scan_rows', ptr(nm), b, ptr(offm), s)
            self.err.check('make_data frames %d-%d' % (f0, f0 + b - 1))
            t1, tm = int(off1[b].item()), int(offm[b].item())
            po = torch.empty(max(1, t1), dtype=torch.int32, device=dev)
            pm = torch.empty(max(1, tm), dtype=torch.int32, device=dev)
            cm = torch.empty(max(1, tm), dtype=torch.int32, device=dev)
            call('rspi_sim_sparse_fill', ptr(counts), b, npix, ptr(off1), ptr(offm), ptr(po),
                 ptr(pm), ptr(cm), s)
            lists['ones'].append(n1[:b].cpu().numpy())
            lists['multi'].append(nm[:b].cpu().numpy())
            lists['place_ones'].append(po[:t1].cpu().numpy())
            lists['place_multi'].append(pm[:tm].cpu().numpy())
            cmh = cm[:tm].cpu().numpy()
            lists['count_multi'].append(cmh)
            photons += t1 + int(cmh.sum(dtype=np.int64))
            sys.stderr.write('\rWritten %d/%d frames (%d)' % (f0 + b, n, photons))
        etime = time.time()
        sys.stderr.write('\nTime taken (make_data): %f s\n' % (etime - stime))
        out.update({k: (np.concatenate(v) if v else np.zeros(0)).astype('i4')
                    for k, v in lists.items()})
        delete = ['ones', 'multi', 'place_ones', 'place_multi', 'count_multi', 'num_pix',
                  'true_shifts', 'true_diameters', 'true_angles', 'bg', 'scale']
        if self.object_hetro:
            delete.append('true_wobbles')
        photonfile.update_datasets(self.out_photons_file, out, delete=delete)
        return out


def main():
    parser = argparse.ArgumentParser(description='Padman data generator')
    parser.add_argument('-c', '--config_file',
                        help='Path to config file (Default: make_data_config.ini)',
                        default='make_data_config.ini')
    parser.add_argument('-m', '--mask_only',
                        help='Create mask only and not the data frames',
                        action='store_true', default=False)
    parser.add_argument('-d', '--data_only',
                        help='Generate data only. Use preexisting mask in file',
                        action='store_true', default=False)
    parser.add_argument('-D', '--device',
                        help='Device number (default: 0)', type=int, default=0)
    args = parser.parse_args()

    torch.cuda.set_device(args.device)
    datagen = DataGenerator(args.config_file)
    if not args.data_only:
        datagen.make_obj()
    if not args.mask_only:
        datagen.make_data(parse=args.data_only)


if __name__ == '__main__':
    main()
