"""HDF5 subset codec (rspi/h5lite.py): round trips and structure.

No HDF5 library exists on this platform, so these tests check the writer
against the reader and the on-disk structures against the format
specification's fixed fields; they cannot compare with libhdf5."""
import struct

import numpy as np
import pytest

from rspi import h5lite
from rspi.photonfile import PhotonsFile, write_photons


def _roundtrip(tmp_path, data):
    path = str(tmp_path / 'f.h5')
    h5lite.write_datasets(path, data)
    return path, h5lite.read_datasets(path)


def test_scalar_types_and_shapes(tmp_path):
    rng = np.random.default_rng(0)
    data = {'i4': rng.integers(-5, 5, 7).astype('<i4'), 'i8': np.array([101 * 101]),
            'u2': rng.integers(0, 60000, (3, 4)).astype('<u2'), 'f8': rng.random((5, 3)),
            'f4': rng.random(9).astype('<f4'), 'c16': rng.random(6) + 1j * rng.random(6),
            'empty': np.zeros(0, 'f8'), 'scalar_like': np.array([3.5])}
    _, back = _roundtrip(tmp_path, data)
    assert sorted(back) == sorted(data)
    for k, v in data.items():
        assert back[k].dtype == v.dtype, k
        np.testing.assert_array_equal(back[k], v)


def test_many_datasets_use_several_symbol_nodes(tmp_path):
    data = {'d%02d' % i: np.arange(i + 1, dtype='<i4') for i in range(30)}
    _, back = _roundtrip(tmp_path, data)
    assert sorted(back) == sorted(data)
    for k, v in data.items():
        np.testing.assert_array_equal(back[k], v)


def test_vlen_lists_with_empty_rows(tmp_path):
    lens = np.array([3, 0, 5, 0, 1])
    flat = np.arange(lens.sum(), dtype='<i4') * 7
    path, back = _roundtrip(tmp_path, {'place_ones': ('vlen', flat, lens)})
    np.testing.assert_array_equal(back['place_ones@flat'], flat)
    np.testing.assert_array_equal(back['place_ones@lens'], lens)


def test_structure_matches_specification(tmp_path):
    path, _ = _roundtrip(tmp_path, {'a': np.arange(3, dtype='<i4')})
    b = open(path, 'rb').read()
    assert b[:8] == b'\x89HDF\r\n\x1a\n'
    assert b[8] == 0 and b[13] == 8 and b[14] == 8           # superblock v0, 8-byte sizes
    leaf_k, int_k = struct.unpack_from('<HH', b, 16)
    assert (leaf_k, int_k) == (4, 16)
    eof = struct.unpack_from('<Q', b, 40)[0]
    assert eof == len(b)
    root = struct.unpack_from('<Q', b, 64)[0]
    assert b[root] == 1                                       # v1 object header
    btree, heap = struct.unpack_from('<QQ', b, 80)
    assert b[btree:btree + 4] == b'TREE' and b[heap:heap + 4] == b'HEAP'


def test_photons_file_h5_and_npz_agree(tmp_path):
    from helpers import random_photons
    d = random_photons(21, 12, 300., 1, empty_frames=(3,))
    for name in ('p.h5', 'p.npz'):
        path = str(tmp_path / name)
        write_photons(path, d)
        f = PhotonsFile(path)
        assert np.array_equal(f['num_pix'], d['num_pix'])
        for key in ('ones', 'multi'):
            np.testing.assert_array_equal(f[key], d[key])
        for key, lens in (('place_ones', d['ones']), ('place_multi', d['multi']),
                          ('count_multi', d['multi'])):
            flat, ln = f.flat(key)
            np.testing.assert_array_equal(flat, d[key])
            np.testing.assert_array_equal(ln, lens)


def test_dataset_reader_rejects_pixel_mismatch(tmp_path):
    from helpers import random_photons
    import dset
    d = random_photons(21, 4, 100., 2)
    path = str(tmp_path / 'p.h5')
    write_photons(path, d)
    host = dset.read_photons(path, 21 * 21)
    np.testing.assert_array_equal(host['place_ones'], d['place_ones'])
    with pytest.raises(AttributeError):
        dset.read_photons(path, 20 * 20)


def test_not_hdf5(tmp_path):
    p = tmp_path / 'x.h5'
    p.write_bytes(b'not an hdf5 file at all')
    with pytest.raises(h5lite.H5FormatError):
        h5lite.read_datasets(str(p))


def test_vlen_beyond_one_global_heap_collection(tmp_path):
    """More than 65,535 non-empty variable-length rows (the 16-bit object
    index of one global heap collection) go to several collections and read
    back in order."""
    from rspi import h5lite
    n = 70000
    rng = np.random.default_rng(4)
    lens = rng.integers(0, 4, n)
    flat = rng.integers(0, 1 << 20, int(lens.sum())).astype('<i4')
    path = str(tmp_path / 'big.h5')
    h5lite.write_datasets(path, {'place_ones': ('vlen', flat, lens), 'ones': lens.astype('i4')})
    out = h5lite.read_datasets(path)
    assert np.array_equal(out['place_ones@flat'], flat)
    assert np.array_equal(out['place_ones@lens'], lens)
    assert np.array_equal(out['ones'], lens)
