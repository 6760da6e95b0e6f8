"""The seeded synthetic-data generator (CPU): photon-file layout invariants,
determinism, conformations and uneven per-frame loads."""
import numpy as np

from oracle import emc_oracle as E

SIZE = 61


def _gen(**kw):
    from rspi import synth
    base = dict(size=SIZE, num_data=300, mean_count=400., n_blobs=10, obj_radius=8.,
                fluence_sigma=0.5, dia=(6., 8.), shift_max=3., seed=7)
    base.update(kw)
    return synth.generate(**base)


def _frame_totals(d):
    starts = np.r_[0, np.cumsum(d['multi'])[:-1]]
    multi = np.add.reduceat(d['count_multi'], starts) if d['count_multi'].size else 0
    multi = np.where(d['multi'] > 0, multi, 0)
    return d['ones'] + multi


def test_layout_and_determinism():
    a, b = _gen(), _gen()
    for k in ('ones', 'multi', 'place_ones', 'place_multi', 'count_multi'):
        assert np.array_equal(a[k], b[k]), k
    assert a['ones'].sum() == a['place_ones'].size
    assert a['multi'].sum() == a['place_multi'].size == a['count_multi'].size
    assert np.all(a['count_multi'] >= 2)
    # pixels ascending within each frame, inside the detector
    off = np.r_[0, np.cumsum(a['ones'])]
    for d in range(a['ones'].size):
        p = a['place_ones'][off[d]:off[d + 1]]
        assert np.all(np.diff(p) > 0)
    assert a['place_ones'].max() < SIZE * SIZE and a['place_ones'].min() >= 0
    ds = E.parse_photons(a['ones'], a['multi'], a['place_ones'], a['place_multi'],
                         a['count_multi'], SIZE * SIZE, True)
    assert abs(ds['mean_count'] - 400.) < 40.
    assert 'true_modes' not in a and a['solution'].shape == (SIZE, SIZE)


def test_conformations():
    from rspi import synth
    d = _gen(num_data=2000, n_modes=3, mode_weights=(0.5, 0.3, 0.2))
    frac = np.bincount(d['true_modes'], minlength=3) / 2000.
    assert np.allclose(frac, (0.5, 0.3, 0.2), atol=0.04)
    assert d['solution'].shape == (3, SIZE, SIZE) and d['fsample'].shape == (3, SIZE * SIZE)
    # conformation m moves 15% of the blobs by 2-4 px and keeps the rest
    rng = np.random.default_rng(1)
    b0 = synth.make_blobs(SIZE, 40, 8., rng)
    b1 = synth.displaced_blobs(b0, 0.15, (2., 4.), rng)
    moved = np.flatnonzero(np.any(b0[:, :2] != b1[:, :2], axis=1))
    assert moved.size == 6
    dist = np.hypot(*(b1[moved, :2] - b0[moved, :2]).T)
    assert np.all((dist >= 2.) & (dist <= 4.))
    assert np.array_equal(b0[:, 2:], b1[:, 2:])
    # the first conformation is the single-mode object of the same seed
    assert np.array_equal(d['solution'][0], _gen(num_data=2000)['solution'])


def test_uneven_loads():
    d = _gen(num_data=400, mean_count=None, count_lognormal=(500., 1.15, 50., 5000.))
    tot = _frame_totals(d)
    target = d['scale']           # each frame's target count / the mean target
    # photon totals follow each frame's own draw (rank correlation), spanning decades
    r = np.corrcoef(np.argsort(np.argsort(tot)), np.argsort(np.argsort(target)))[0, 1]
    assert r > 0.95
    assert tot.max() / max(1, tot.min()) > 20
    assert tot.max() <= 5000 * 1.2
