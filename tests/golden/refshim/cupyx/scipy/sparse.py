"""Stand-in for cupyx.scipy.sparse.csr_matrix on top of SciPy.

Two-array indexing ``m[rows, cols]`` returns a dense (1, n) array, as cupyx
does (scipy would return an np.matrix).
"""
import numpy as np
from scipy import sparse as _sp

import cupy as _cp


class csr_matrix:
    def __init__(self, arg, shape=None):
        if _sp.issparse(arg):
            self._m = arg.tocsr()
        else:
            data, indices, indptr = arg
            self._m = _sp.csr_matrix((np.asarray(data), np.asarray(indices),
                                      np.asarray(indptr)), shape=shape)

    @property
    def shape(self):
        return self._m.shape

    def __add__(self, other):
        return csr_matrix(self._m + other._m)

    def __getitem__(self, key):
        if (isinstance(key, tuple) and len(key) == 2
                and all(isinstance(k, np.ndarray) for k in key)):
            rows, cols = (np.asarray(k).view(np.ndarray) for k in key)
            vals = np.asarray(self._m[rows, cols]).ravel()
            return np.expand_dims(vals, 0).view(_cp.ndarray)
        res = self._m[key]
        return csr_matrix(res) if _sp.issparse(res) else res

    def transpose(self):
        return csr_matrix(self._m.transpose())

    def tocsr(self):
        return csr_matrix(self._m.tocsr())

    def sum(self, axis=None):
        return np.asarray(self._m.sum(axis))

    def toarray(self):
        return self._m.toarray().view(_cp.ndarray)
