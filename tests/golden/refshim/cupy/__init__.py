"""NumPy-backed stand-in for the parts of CuPy the reference uses.

Arrays are a NumPy subclass with CuPy's ``.get()``; every NumPy function
reached through this module returns that subclass.  ``RawModule`` runs the
reference's own kernels.cu compiled for the CPU (oracle/_ref).  Test
infrastructure for tests/golden/make_golden.py only.
"""
import ctypes
import os

import numpy as _np

from . import cuda  # noqa: F401  (cp.cuda.*)

pi = _np.pi
bool_ = _np.bool_
float64 = _np.float64
complex128 = _np.complex128
int32 = _np.int32


class ndarray(_np.ndarray):
    def get(self):
        return _np.array(self, copy=True).view(_np.ndarray)


def _wrap(obj):
    if isinstance(obj, _np.ndarray) and not isinstance(obj, ndarray):
        return obj.view(ndarray)
    if isinstance(obj, tuple):
        return tuple(_wrap(o) for o in obj)
    if isinstance(obj, list):
        return [_wrap(o) for o in obj]
    return obj


def _unwrap(obj):
    if isinstance(obj, ndarray):
        return obj.view(_np.ndarray)
    if isinstance(obj, (list, tuple)):
        return type(obj)(_unwrap(o) for o in obj)
    return obj


def __getattr__(name):
    attr = getattr(_np, name)
    if callable(attr) and not isinstance(attr, type):
        def fn(*args, **kwargs):
            return _wrap(attr(*[_unwrap(a) for a in args],
                              **{k: _unwrap(v) for k, v in kwargs.items()}))
        return fn
    return attr


def array(obj, dtype=None, copy=True):
    if hasattr(obj, 'toarray'):          # scipy matrix results
        obj = _np.asarray(obj)
    return _np.array(_unwrap(obj), dtype=dtype, copy=copy).view(ndarray)


def asarray(obj, dtype=None):
    return _np.asarray(_unwrap(obj), dtype=dtype).view(ndarray)


def get_default_memory_pool():
    class _Pool:
        def used_bytes(self):
            return 0
    return _Pool()


# ---------------------------------------------------------------------------
# RawModule: reference kernels compiled for the CPU
# ---------------------------------------------------------------------------
_REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), '..', '..', '..', '..'))
_LIB_PATH = os.path.join(_REPO, 'oracle', '_ref', 'libref_kernels_cpu.so')
_lib = None

_P = ctypes.c_void_p
_D = ctypes.c_double
_L = ctypes.c_longlong
_U = ctypes.c_uint

# name -> (launcher, grid dims, argument kinds)
#   'p:<dtype>' pointer to a contiguous array of that dtype, 'd' double, 'l' long long
_SIGS = {
    'slice_gen': ('ref_slice_gen', 2, ['p:f8', 'd', 'd', 'l', 'p:f8', 'l', 'p:f8']),
    'slice_gen_holo': ('ref_slice_gen_holo', 2,
                       ['p:c16', 'd', 'd', 'd', 'd', 'd', 'l', 'p:f8', 'l', 'p:f8']),
    'slice_merge': ('ref_slice_merge', 2, ['p:f8', 'd', 'l', 'p:f8', 'p:f8']),
    'calc_prob_all': ('ref_calc_prob_all', 1,
                      ['p:f8', 'p:i4', 'l', 'p:i4', 'p:i4', 'p:i8', 'p:i8', 'p:i4',
                       'p:i4', 'p:i4', 'd', 'p:f8', 'p:f8']),
    'merge_all': ('ref_merge_all', 1,
                  ['p:f8', 'l', 'p:i4', 'p:i4', 'p:i8', 'p:i8', 'p:i4', 'p:i4',
                   'p:i4', 'p:f8']),
    'get_f_dt': ('ref_get_f_dt', 1, ['p:c16', 'p:c16', 'l', 'l', 'p:c16']),
}


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError('build oracle/_ref first: python oracle/ref_cpu/build.py')
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


class _Unused:
    """Kernels fetched by the reference but never launched on its run path."""

    def __init__(self, name):
        self.name = name

    def __call__(self, *args):
        raise NotImplementedError('kernel %s is not on the reference run path' % self.name)


class _Kernel:
    def __init__(self, name):
        self.name = name
        self.launcher, self.ndim, self.kinds = _SIGS[name]
        fn = getattr(_load(), self.launcher)
        fn.restype = None
        fn.argtypes = [_U] * (2 * self.ndim) + [
            _P if k.startswith('p') else (_D if k == 'd' else _L) for k in self.kinds]
        self.fn = fn

    def __call__(self, grid, block, args):
        assert len(args) == len(self.kinds), self.name
        cargs = []
        for a, k in zip(args, self.kinds):
            if k.startswith('p'):
                arr = _np.asarray(a)
                want = _np.dtype(k[2:])
                if arr.dtype != want or not arr.flags['C_CONTIGUOUS']:
                    raise TypeError('%s: argument needs contiguous %s, got %s' %
                                    (self.name, want, arr.dtype))
                cargs.append(arr.ctypes.data)
            elif k == 'd':
                cargs.append(float(a))
            else:
                cargs.append(int(a))
        dims = [int(g) for g in grid] + [int(b) for b in block]
        if self.ndim == 2:
            dims = [dims[0], dims[1], dims[2], dims[3]]
        self.fn(*dims, *cargs)


class RawModule:
    def __init__(self, code=None, **kwargs):
        self.code = code

    def get_function(self, name):
        return _Kernel(name) if name in _SIGS else _Unused(name)
