"""Photons-file container with the reference's dataset names.

The reference stores sparse photons in HDF5 (make_data.py:245-251):
``num_pix`` (1,), ``ones`` / ``multi`` int32 (N), and the vlen int32 lists
``place_ones``, ``place_multi``, ``count_multi`` (N), plus optional ``bg``
and truth datasets.  h5py is not available on this platform, so the same
datasets are kept in an ``.npz`` container: a vlen dataset ``name`` is stored
as ``name@flat`` (the concatenated int32 values) and ``name@lens`` (per-row
lengths).  ``.h5`` paths go through the HDF5 subset codec in ``h5lite``.
"""
import os

import numpy as np

VLEN = ('place_ones', 'place_multi', 'count_multi')


def write_photons(path, data):
    """Write ``data`` (flat arrays as produced by ``synth.generate``)."""
    if path.endswith('.h5'):
        from . import h5lite
        return h5lite.write_photons(path, data)
    out = {}
    lens = {'place_ones': data['ones'], 'place_multi': data['multi'],
            'count_multi': data['multi']}
    for key, val in data.items():
        if key in VLEN:
            out[key + '@flat'] = np.asarray(val, dtype='i4')
            out[key + '@lens'] = np.asarray(lens[key], dtype='i8')
        else:
            out[key] = np.asarray(val)
    tmp = path + '.tmp'
    with open(tmp, 'wb') as fh:
        np.savez(fh, **out)
    os.replace(tmp, path)
    return path


def sparse_from_dense(frames):
    """ones/multi lists of dense (N, P) counts, frames in order and pixels
    ascending within a frame (the make_data.py:323-328 layout)."""
    f = np.asarray(frames)
    one, many = f == 1, f > 1
    _, po = np.nonzero(one)
    dm, pm = np.nonzero(many)
    return dict(ones=one.sum(1).astype('i4'), multi=many.sum(1).astype('i4'),
                place_ones=po.astype('i4'), place_multi=pm.astype('i4'),
                count_multi=f[dm, pm].astype('i4'))


class PhotonsFile:
    """Read access with h5py-like semantics: ``f['ones'][:]``,
    ``f['place_ones'].shape``, ``KeyError`` for a missing dataset."""

    def __init__(self, path):
        self.path = path
        if path.endswith('.h5'):
            from . import h5lite
            self._raw = h5lite.read_datasets(path)
        else:
            with np.load(path) as z:
                self._raw = {k: z[k] for k in z.files}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return None

    def __contains__(self, key):
        return key in self._raw or key + '@flat' in self._raw

    def num_rows(self, key):
        if key + '@lens' in self._raw:
            return self._raw[key + '@lens'].shape[0]
        return self._raw[key].shape[0]

    def flat(self, key):
        """Concatenated values of a vlen dataset and its per-row lengths."""
        if key + '@flat' in self._raw:
            return self._raw[key + '@flat'], self._raw[key + '@lens']
        raise KeyError(key)

    def __getitem__(self, key):
        if key in self._raw:
            return self._raw[key]
        raise KeyError(key)
