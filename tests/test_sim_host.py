"""Host side of the data simulator on CPU: the photons-file update that
stands in for h5py's append mode, and the simulator oracle's own
consistency (normalisation, sparse lists)."""
import numpy as np
import pytest

from oracle import emc_oracle as E
from oracle import sim_oracle as S


@pytest.mark.parametrize('ext', ['.h5', '.npz'])
def test_update_datasets_keeps_other_datasets(tmp_path, ext):
    from rspi import photonfile
    path = str(tmp_path / ('p' + ext))
    photonfile.update_datasets(path, {'solution': np.arange(16.).reshape(4, 4)})
    frames = dict(ones=np.array([1, 0, 2], 'i4'), multi=np.array([0, 1, 1], 'i4'),
                  place_ones=np.array([3, 4, 5], 'i4'), place_multi=np.array([7, 8], 'i4'),
                  count_multi=np.array([2, 3], 'i4'), num_pix=np.array([16]),
                  true_shifts=np.ones((3, 2)))
    photonfile.update_datasets(path, frames)
    f = photonfile.PhotonsFile(path)
    assert np.array_equal(f['solution'], np.arange(16.).reshape(4, 4))
    po, lens = f.flat('place_ones')
    assert np.array_equal(po, [3, 4, 5]) and np.array_equal(lens, [1, 0, 2])
    cm, lm = f.flat('count_multi')
    assert np.array_equal(cm, [2, 3]) and np.array_equal(lm, [0, 1, 1])
    assert f['true_shifts'].shape == (3, 2)
    # a later update replaces the frames and drops what it is told to
    photonfile.update_datasets(path, dict(ones=np.array([1], 'i4'), multi=np.array([0], 'i4'),
                                          place_ones=np.array([9], 'i4'),
                                          place_multi=np.zeros(0, 'i4'),
                                          count_multi=np.zeros(0, 'i4')),
                               delete=['true_shifts'])
    f = photonfile.PhotonsFile(path)
    assert 'true_shifts' not in f and 'solution' in f
    assert np.array_equal(f.flat('place_ones')[0], [9])
    with pytest.raises(ValueError):
        photonfile.update_datasets(path, dict(place_ones=np.array([1], 'i4')))


def test_sparse_lists_two_ways():
    rng = np.random.default_rng(5)
    frames = rng.poisson(0.4, (23, 50)).astype('i4')
    frames[3] = 0
    from rspi.photonfile import sparse_from_dense
    a = S.sparse_lists(frames)
    b = sparse_from_dense(frames)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_expected_frame_normalisation():
    """Before the rotation a frame holds mean_count photons on the detector
    mask; with angle 0 the rotation keeps every pixel whose footprint stays
    on the detector."""
    size = 45
    obj, _ = S.deterministic_object(size)
    model = S.centred_fft(obj).ravel()
    zero = np.zeros(size * size)
    view = E.holo_slice(model, 0.3, -0.2, 7., 50., 1.7, size, zero) * \
        S.detector_mask(size).ravel()
    view *= 500. / view.sum()
    got = S.expected_frame(model, 0.3, -0.2, 7., 50., 1.7, 0., size, 500.)
    x, y = np.indices((size, size))
    inside = ((x <= size - 2) & (y <= size - 2)).ravel()
    np.testing.assert_allclose(got[inside], view[inside], rtol=1e-13, atol=1e-15)
    assert np.all(got[~inside] == 0.)
    assert abs(view.sum() - 500.) < 1e-9
    # a heterogeneous object's two masks double the view before the
    # normalisation, which cancels it
    got2 = S.expected_frame(model, 0.3, -0.2, 7., 50., 1.7, 0., size, 500., hetro=True)
    np.testing.assert_allclose(got2, got, rtol=1e-13, atol=1e-15)


def test_frame_models():
    size = 31
    obj, wob = S.deterministic_object(size, hetro=True)
    m, w = S.centred_fft(obj), S.centred_fft(wob)
    assert np.array_equal(S.frame_model('iso', m, w, 0, 4.5, size), m)
    qx, qy = S.qvals(size)
    a = w * np.exp(2j * np.pi * 4.5 * (qx + qy))
    b = np.fliplr(w * np.exp(2j * np.pi * (qx * 4.5 + (-3.7) * qy * 4.5)))
    tol = dict(rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(S.frame_model('mix', m, w, 2, 4.5, size), m + a, **tol)
    np.testing.assert_allclose(S.frame_model('mix', m, w, 3, 4.5, size), m + b, **tol)
    np.testing.assert_allclose(S.frame_model('homo', m, w, 3, 4.5, size), m + (a + b) / 2, **tol)
    with pytest.raises(ValueError):
        S.frame_model('other', m, w, 0, 1., size)
