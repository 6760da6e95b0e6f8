"""Sparse photon dataset on the GPU -- drop-in for the reference ``dset.py``.

``Dataset(photons_file, num_pix, need_scaling=False)`` keeps the reference's
attributes (dset.py:16-61): ``num_data``, ``ones``, ``multi``,
``ones_accum``, ``multi_accum`` (int64 exclusive prefix sums),
``place_ones``, ``place_multi``, ``count_multi``, ``mean_count``,
``counts`` (when ``need_scaling``), ``bg``, ``mem``, plus ``get_frame`` and
``get_powder``.  Arrays are torch CUDA tensors instead of CuPy arrays; the
prefix sums, counts and powder are computed by librspi kernels.  A photons
file may also hold dense uint16 counts ``frames`` (N, num_pix) for the
dense likelihood form; a file with only ``frames`` gets its sparse lists
derived from them.

With ``shard=True`` inside an initialised torch.distributed group of several
ranks, the dataset holds this rank's frames only (a contiguous block of the
file's frames, or the whole of ``photons_file.format(rank=rank)`` when the
name contains ``{rank}``); ``num_data`` counts them and ``num_data_global``
all frames, and the mean count, scales and powder are the whole dataset's.
"""
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from rspi.device import DevicePhotons  # noqa: E402
from rspi.shard import shard_photons  # noqa: E402
from rspi.shard import world as shard_world  # noqa: E402
from rspi.photonfile import PhotonsFile, sparse_from_dense  # noqa: E402


def read_photons(photons_file, num_pix=None):
    """Host arrays of a photons file (dset.py:23-60 reads).  Raises
    AttributeError when ``num_pix`` does not match (dset.py:24-25)."""
    with PhotonsFile(photons_file) as fptr:
        if num_pix is not None and np.any(num_pix != np.asarray(fptr['num_pix'])):
            raise AttributeError('Number of pixels in photons file does not match')
        frames = np.asarray(fptr['frames'], dtype=np.uint16) if 'frames' in fptr else None
        npix = int(np.asarray(fptr['num_pix']).ravel()[0])
        if frames is not None and 'place_ones' not in fptr:
            # dense-only file: the sparse lists are derived from the frames
            host = sparse_from_dense(frames)
            host.update(num_data=frames.shape[0], num_pix=npix, frames=frames,
                        bg=np.asarray(fptr['bg'], dtype='f8').ravel() if 'bg' in fptr else None)
            return host
        num_data = fptr.num_rows('place_ones')
        po, po_len = fptr.flat('place_ones')
        pm, pm_len = fptr.flat('place_multi')
        cm, _ = fptr.flat('count_multi')
        try:
            ones = np.asarray(fptr['ones']).astype('i4')
        except KeyError:
            ones = po_len.astype('i4')
        try:
            multi = np.asarray(fptr['multi']).astype('i4')
        except KeyError:
            multi = pm_len.astype('i4')
        try:
            bg = np.asarray(fptr['bg'], dtype='f8').ravel()
        except KeyError:
            bg = None
    return dict(num_data=num_data, num_pix=npix, ones=ones, multi=multi, place_ones=po,
                place_multi=pm, count_multi=cm, bg=bg, frames=frames)


class Dataset():
    '''Parses sparse photons dataset from a photons file onto the GPU

    Args:
        photons_file (str): Path to photons file (.npz container or .h5)
        num_pix (int): Expected number of pixels in sparse file
        need_scaling (bool, optional): Whether scaling will be used
        device (optional): CUDA device (default: current)
    '''
    def __init__(self, photons_file, num_pix, need_scaling=False, device=None, num_data=-1,
                 shard=False):
        self.powder = None
        self.photons_file = photons_file
        self.num_pix = num_pix
        rank, size = shard_world() if shard else (0, 1)
        pre_sharded = size > 1 and '{rank}' in photons_file
        if pre_sharded:
            # one file per rank (frames already split)
            photons_file = photons_file.format(rank=rank)
        host = read_photons(photons_file, num_pix)
        if 0 <= num_data < host['num_data']:
            host = _first_frames(host, num_data)
        before = torch.cuda.memory_allocated() if torch.cuda.is_available() else 0
        if size > 1:
            # this rank's frames, with the dataset-wide mean count and powder
            self.photons = shard_photons(host, num_pix, need_scaling, device,
                                         pre_sharded=pre_sharded)
            self.num_data_global = self.photons.num_data_global
        else:
            self.photons = DevicePhotons(host['ones'], host['multi'], host['place_ones'],
                                         host['place_multi'], host['count_multi'], num_pix,
                                         need_scaling, device, frames=host.get('frames'))
            self.num_data_global = self.photons.num_data
        ph = self.photons
        self.num_data = ph.num_data
        self.device = ph.device
        self.ones, self.multi = ph.ones, ph.multi
        self.ones_accum, self.multi_accum = ph.ones_accum, ph.multi_accum
        self.place_ones, self.place_multi, self.count_multi = ph.place_ones, ph.place_multi, ph.count_multi
        self.mean_count = ph.mean_count
        if need_scaling:
            self.counts = ph.counts
        if host['bg'] is not None:
            self.bg = torch.from_numpy(host['bg']).to(self.device)
            print('Using background model with %.2f photons/frame' % float(host['bg'].sum()))
        else:
            self.bg = torch.zeros(self.num_pix, dtype=torch.float64, device=self.device)
        self.mem = torch.cuda.memory_allocated() - before

    def get_frame(self, num):
        """Get particular frame from photons_file (dset.py:63-72)"""
        o_a = int(self.ones_accum[num])
        m_a = int(self.multi_accum[num])
        frame = torch.zeros(self.num_pix, dtype=torch.int32, device=self.device)
        po = self.place_ones[o_a:o_a + int(self.ones[num])].long()
        frame.index_add_(0, po, torch.ones_like(po, dtype=torch.int32))
        pm = self.place_multi[m_a:m_a + int(self.multi[num])].long()
        frame.index_add_(0, pm, self.count_multi[m_a:m_a + int(self.multi[num])])
        return frame

    def get_powder(self):
        """Mean photons per pixel over frames (dset.py:74-83), computed on the GPU"""
        if self.powder is None:
            self.powder = self.photons.powder
        return self.powder


def _first_frames(host, n):
    """The first ``n`` frames of a host photon dict (maxLP.py:55-58 ``num_data``)."""
    o_end = int(host['ones'][:n].sum())
    m_end = int(host['multi'][:n].sum())
    out = dict(host)
    out.update(num_data=n, ones=host['ones'][:n], multi=host['multi'][:n],
               place_ones=host['place_ones'][:o_end], place_multi=host['place_multi'][:m_end],
               count_multi=host['count_multi'][:m_end])
    if host.get('frames') is not None:
        out['frames'] = host['frames'][:n]
    return out
