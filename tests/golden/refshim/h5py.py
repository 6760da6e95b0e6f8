"""Stand-in for h5py over .npz containers (test infrastructure).

A vlen dataset ``name`` is stored as ``name@flat`` + ``name@lens`` and read
back as an object array of int32 arrays, as h5py returns it.
"""
import numpy as np


class _Dataset:
    def __init__(self, value):
        self._v = value

    @property
    def shape(self):
        return self._v.shape

    def __getitem__(self, key):
        if key is Ellipsis:
            return np.array(self._v)
        return self._v[key]


class File:
    def __init__(self, name, mode='r'):
        self.name = name
        self.mode = mode
        self._data = {}
        if mode in ('r', 'a', 'r+'):
            try:
                with np.load(name) as z:
                    raw = {k: z[k] for k in z.files}
            except FileNotFoundError:
                if mode == 'r':
                    raise
                raw = {}
            for key, val in raw.items():
                if key.endswith('@flat'):
                    base = key[:-5]
                    lens = raw[base + '@lens']
                    bounds = np.concatenate([[0], np.cumsum(lens)])
                    arr = np.empty(len(lens), dtype=object)
                    for i in range(len(lens)):
                        arr[i] = val[bounds[i]:bounds[i + 1]].astype('i4')
                    self._data[base] = arr
                elif not key.endswith('@lens'):
                    self._data[key] = val

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __contains__(self, key):
        return key in self._data

    def __getitem__(self, key):
        if key not in self._data:
            raise KeyError(key)
        return _Dataset(self._data[key])

    def __setitem__(self, key, value):
        self._data[key] = np.asarray(value)

    def __delitem__(self, key):
        del self._data[key]

    def close(self):
        if self.mode == 'r':
            return
        out = {}
        for key, val in self._data.items():
            if val.dtype == object:
                out[key + '@flat'] = np.concatenate([np.asarray(v, dtype='i4') for v in val]) \
                    if len(val) else np.zeros(0, 'i4')
                out[key + '@lens'] = np.array([len(v) for v in val], dtype='i8')
            else:
                out[key] = val
        with open(self.name, 'wb') as fh:
            np.savez(fh, **out)
