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


def update_datasets(path, new, delete=()):
    """Write the datasets ``new`` into the photons file ``path`` (HDF5 for
    ``.h5``, else ``.npz``), keeping the file's other datasets except those
    named in ``delete`` -- what the reference does with h5py's append mode
    (make_data.py:156-167, 228-276).  Values of ``place_ones``,
    ``place_multi`` and ``count_multi`` are flat arrays whose row lengths are
    ``ones`` / ``multi`` (as for ``write_photons``)."""
    raw = {}
    if os.path.exists(path):
        raw = dict(PhotonsFile(path)._raw)
    gone = set(delete) | set(new)
    raw = {k: v for k, v in raw.items() if k.split('@')[0] not in gone}
    lens = {'place_ones': 'ones', 'place_multi': 'multi', 'count_multi': 'multi'}
    for key, val in new.items():
        if key in VLEN:
            src = new.get(lens[key])
            if src is None:
                raise ValueError('%s needs %s in the same update' % (key, lens[key]))
            raw[key + '@flat'] = np.asarray(val, dtype='i4')
            raw[key + '@lens'] = np.asarray(src, dtype='i8')
        else:
            raw[key] = np.asarray(val)
    if path.endswith('.h5'):
        from . import h5lite
        out = {}
        for k, v in raw.items():
            if k.endswith('@flat'):
                name = k[:-5]
                out[name] = ('vlen', np.asarray(v, dtype='<i4'), raw[name + '@lens'])
            elif not k.endswith('@lens'):
                out[k] = v
        h5lite.write_datasets(path, out)
        return path
    tmp = path + '.tmp'
    with open(tmp, 'wb') as fh:
        np.savez(fh, **raw)
    os.replace(tmp, path)
    return path
