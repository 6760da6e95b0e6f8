"""The data simulator on the GPU (make_data.py's per-frame loop as batched
kernels, csrc/simulate.cu; the drop-in DataGenerator, make_data.py).

* expected counts of every frame (frame model of each object type,
  holographic intensity, mask, normalisation, rotation, background) against
  the FP64 oracle (make_data.py:294-322) and against the same steps run
  with the reference's own kernels (slice_gen_holo, slice_gen from
  kernels.cu, built by oracle/ref_gpu/build.py): within 1e-12 of the
  frame's largest value;
* the Poisson sampler: mean, variance and a chi-square test of the law for
  means from 0.02 to 2,000 (both the inversion and the rejection branch);
* the sparse lists (ones / multi / place_* / count_multi) exactly those of
  the counts (make_data.py:324-328); counts independent of the batching;
* DataGenerator end to end: the deterministic object bit-compatible with
  the oracle's, the file's datasets and shapes, photons per frame near
  mean_count, a seeded configuration reproducing its file, and EMC reading
  the file."""
import numpy as np
import pytest
import torch

from oracle import sim_oracle as S

pytestmark = pytest.mark.gpu


def _call(name, *args):
    from rspi.lib import call
    call(name, *args)


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to('cuda', dtype)


def _frames(kind, size, n, hetro, bg, seed, frame0=0, batch=None):
    """(expected, counts, params) from the librspi kernels for n frames."""
    from rspi.device import ErrorWord, cur_stream, ptr
    rng = np.random.default_rng(seed)
    obj, wob = S.deterministic_object(size, hetro)
    model = _dev(S.centred_fft(obj).ravel(), torch.complex128)
    wmod = _dev(S.centred_fft(wob).ravel(), torch.complex128) if hetro else None
    shifts = rng.standard_normal((n, 2)) * 0.7
    dia = rng.standard_normal(n) * 0.5 + 7.
    scale = rng.gamma(2., 0.5, n)
    ang = rng.random(n) * 2 * np.pi
    w = rng.standard_normal(n) * 0.8 if kind == 'blur' else np.full(n, 4.5)
    bgv = rng.random(size * size) * 0.01 if bg else None
    npix = size * size
    view = torch.empty((n, npix), dtype=torch.float64, device='cuda')
    exp = torch.empty((n, npix), dtype=torch.float64, device='cuda')
    counts = torch.empty((n, npix), dtype=torch.int32, device='cuda')
    err = ErrorWord('cuda')
    kd = dict(iso=0, homo=1, mix=2, blur=3)[kind]
    cs = _dev(np.stack([np.cos(ang), np.sin(ang)], 1).ravel())
    sh, di, sc, wd = _dev(shifts.ravel()), _dev(dia), _dev(scale), _dev(w)
    bgd = _dev(bgv) if bg else None
    batch = batch or n
    for f0 in range(0, n, batch):
        b = min(batch, n - f0)
        _call('rspi_sim_views', ptr(model), ptr(wmod), kd, frame0 + f0, b, ptr(wd[f0:]),
              ptr(sh[2 * f0:]), ptr(di[f0:]), ptr(sc[f0:]), 3.5, 1000., 2. if hetro else 1., size,
              ptr(view[f0:]), ptr(err.t), cur_stream())
        _call('rspi_sim_counts', ptr(view[f0:]), frame0 + f0, b, ptr(cs[2 * f0:]), ptr(bgd), size,
              12345, ptr(counts[f0:]), ptr(exp[f0:]), ptr(err.t), cur_stream())
    torch.cuda.synchronize()
    err.check('simulator')
    params = dict(obj=obj, wob=wob, shifts=shifts, dia=dia, scale=scale, ang=ang, w=w, bg=bgv)
    return exp.cpu().numpy(), counts.cpu().numpy(), params


def _oracle_frame(kind, size, i, p, hetro):
    model = S.centred_fft(p['obj'])
    wmod = S.centred_fft(p['wob']) if hetro else None
    fm = S.frame_model(kind, model, wmod, i, p['w'][i], size)
    return S.expected_frame(fm.ravel(), p['shifts'][i, 0], p['shifts'][i, 1], p['dia'][i], 3.5,
                            p['scale'][i], p['ang'][i], size, 1000., p['bg'], hetro)


@pytest.mark.parametrize('kind,hetro,bg,size', [('iso', False, False, 61), ('iso', False, True, 101),
                                                ('homo', True, False, 61), ('mix', True, True, 61),
                                                ('blur', True, False, 45)])
def test_expected_frames_match_oracle(kind, hetro, bg, size):
    n = 6
    exp, _, p = _frames(kind, size, n, hetro, bg, seed=size)
    for i in range(n):
        want = _oracle_frame(kind, size, i, p, hetro)
        assert np.max(np.abs(exp[i] - want)) <= 1e-12 * np.max(np.abs(want)), (kind, i)


def test_expected_frames_match_reference_kernels():
    """The same frames through the reference's slice_gen_holo and slice_gen
    (kernels.cu:6-82) with make_data.py's grids, the mask and normalisation
    between them as make_data.py:314-318 does them."""
    from oracle.ref_gpu import replay
    lib = replay.load()
    size, n = 61, 4
    for kind, hetro in (('iso', False), ('mix', True)):
        exp, _, p = _frames(kind, size, n, hetro, True, seed=7)
        model = S.centred_fft(p['obj'])
        wmod = S.centred_fft(p['wob']) if hetro else None
        mask = S.detector_mask(size).ravel()
        bm = (size + 31) // 32
        zero = torch.zeros(size * size, dtype=torch.float64, device='cuda')
        bgd = _dev(p['bg'])
        for i in range(n):
            fm = _dev(S.frame_model(kind, model, wmod, i, p['w'][i], size).ravel(),
                      torch.complex128)
            view = torch.empty(size * size, dtype=torch.float64, device='cuda')
            rview = torch.empty_like(view)
            s = torch.cuda.current_stream().cuda_stream
            replay._ok(lib.ref_gpu_slice_gen_holo(
                bm, bm, 32, 32, replay._p(fm), float(p['shifts'][i, 0]), float(p['shifts'][i, 1]),
                float(p['dia'][i]), 3.5, float(p['scale'][i]), size, replay._p(zero), 0,
                replay._p(view), s), 'slice_gen_holo')
            view *= _dev((mask + mask) if hetro else mask)
            view *= 1000. / view.sum()
            replay._ok(lib.ref_gpu_slice_gen(bm, bm, 32, 32, replay._p(view), float(p['ang'][i]),
                                             1., size, replay._p(bgd), 0, replay._p(rview), s),
                       'slice_gen')
            want = rview.cpu().numpy()
            # the reference takes cos / sin of the angle on the device, the
            # simulator from the host: a pixel whose rotated position lies
            # within 1e-9 of the detector's edge may fall on either side
            x, y = np.indices((size, size))
            c = size // 2
            tx = (x - c) * np.cos(p['ang'][i]) - (y - c) * np.sin(p['ang'][i]) + c
            ty = (x - c) * np.sin(p['ang'][i]) + (y - c) * np.cos(p['ang'][i]) + c
            edge = np.zeros((size, size), bool)
            for t in (tx, ty):
                edge |= (np.abs(t) < 1e-9) | (np.abs(t - (size - 1)) < 1e-9)
            ok = ~edge.ravel()
            assert np.max(np.abs(exp[i] - want)[ok]) <= 1e-12 * np.max(np.abs(want)), (kind, i)


@pytest.mark.parametrize('lam', [0.02, 0.7, 3., 9.9, 10., 37.5, 2000.])
def test_poisson_sampler_law(lam):
    """2^21 draws: mean and variance within 6 standard errors, and the
    chi-square statistic of the counts against the Poisson law (bins with an
    expected count of at least 20, the tails pooled) below the 1e-6 quantile."""
    from scipy import stats
    from rspi.device import ErrorWord, cur_stream, ptr
    n = 1 << 21
    lamd = torch.full((n,), lam, dtype=torch.float64, device='cuda')
    out = torch.empty(n, dtype=torch.int32, device='cuda')
    err = ErrorWord('cuda')
    _call('rspi_sim_poisson', ptr(lamd), n, 2026, int(lam * 1000), ptr(out), ptr(err.t),
          cur_stream())
    torch.cuda.synchronize()
    err.check('poisson')
    x = out.cpu().numpy().astype(np.int64)
    assert x.min() >= 0
    se = np.sqrt(lam / n)
    assert abs(x.mean() - lam) <= 6 * se
    # the variance of the sample variance of a Poisson law: (lam + 2 lam^2) / n
    assert abs(x.var() - lam) <= 6 * np.sqrt((lam + 2 * lam * lam) / n)
    k = np.arange(0, int(lam + 12 * np.sqrt(lam) + 20))
    pmf = stats.poisson.pmf(k, lam)
    expct = pmf * n
    keep = expct >= 20
    lo, hi = np.flatnonzero(keep)[0], np.flatnonzero(keep)[-1]
    obs = np.bincount(x, minlength=k.size + 1)[:k.size]
    o = np.concatenate([[obs[:lo + 1].sum()], obs[lo + 1:hi], [n - obs[:hi].sum()]])
    e = np.concatenate([[expct[:lo + 1].sum()], expct[lo + 1:hi], [n - expct[:hi].sum()]])
    chi2 = float(((o - e) ** 2 / e).sum())
    dof = o.size - 1
    assert dof >= 1
    assert chi2 <= stats.chi2.ppf(1 - 1e-6, dof), (chi2, dof)


def test_sparse_lists_and_batching():
    from rspi.device import cur_stream, ptr
    size, n = 45, 37
    exp, counts, _ = _frames('iso', size, n, False, True, seed=3)
    _, counts2, _ = _frames('iso', size, n, False, True, seed=3, batch=10)
    # a frame's draws depend on (seed, frame, pixel) only
    assert np.array_equal(counts, counts2)
    c = _dev(counts, torch.int32)
    npix = size * size
    n1 = torch.empty(n, dtype=torch.int32, device='cuda')
    nm = torch.empty_like(n1)
    o1 = torch.empty(n + 1, dtype=torch.int64, device='cuda')
    om = torch.empty_like(o1)
    _call('rspi_sim_sparse_counts', ptr(c), n, npix, ptr(n1), ptr(nm), cur_stream())
    _call('rspi_scan_rows', ptr(n1), n, ptr(o1), cur_stream())
    _call('rspi_scan_rows', ptr(nm), n, ptr(om), cur_stream())
    t1, tm = int(o1[n]), int(om[n])
    po = torch.full((t1,), -1, dtype=torch.int32, device='cuda')
    pm = torch.full((tm,), -1, dtype=torch.int32, device='cuda')
    cm = torch.full((tm,), -1, dtype=torch.int32, device='cuda')
    _call('rspi_sim_sparse_fill', ptr(c), n, npix, ptr(o1), ptr(om), ptr(po), ptr(pm), ptr(cm),
          cur_stream())
    want = S.sparse_lists(counts)
    assert np.array_equal(n1.cpu().numpy(), want['ones'])
    assert np.array_equal(nm.cpu().numpy(), want['multi'])
    assert np.array_equal(po.cpu().numpy(), want['place_ones'])
    assert np.array_equal(pm.cpu().numpy(), want['place_multi'])
    assert np.array_equal(cm.cpu().numpy(), want['count_multi'])
    # photons per frame near the expectation (Poisson: within 6 sigma)
    tot = counts.sum(1)
    mu = exp.sum(1)
    assert np.all(np.abs(tot - mu) <= 6 * np.sqrt(mu) + 1)


def _config(path, size=61, n=300, kind='iso', hetro=False, random=False, seed=11, bg=None,
            out='photons.h5'):
    text = ('[parameters]\nsize = %d\n[make_data]\nobject_type = %s\nobject_hetro = %s\n'
            'create_random = %s\nnum_data = %d\nmean_count = 2000\ndia_params = 7 0.5\n'
            'shift_sigma = 0.5\nwobble_sigma = 0.5\nrel_scale = 300\nfluence = gamma\n'
            'output_folder = data/\nout_photons_file = %s\nseed = %d\n' %
            (size, kind, 'yes' if hetro else 'no', 'yes' if random else 'no', n, out, seed))
    if bg is not None:
        text += 'bg_count = %g\n' % bg
    with open(path, 'w') as f:
        f.write(text)
    return path


def test_datagenerator_writes_reference_layout(tmp_path):
    from make_data import DataGenerator
    from rspi.photonfile import PhotonsFile
    cfg = _config(str(tmp_path / 'sim.ini'))
    gen = DataGenerator(cfg)
    gen.make_obj()
    obj, _ = S.deterministic_object(61)
    np.testing.assert_allclose(gen.object.cpu().numpy(), obj, rtol=1e-15, atol=1e-15)
    gen.make_data()
    f = PhotonsFile(str(tmp_path / 'photons.h5'))
    n = 300
    for k in ('ones', 'multi', 'true_angles', 'true_diameters', 'scale'):
        assert f[k].shape == (n,), k
    assert f['true_shifts'].shape == (n, 2)
    assert int(f['num_pix'][0]) == 61 * 61
    np.testing.assert_allclose(f['solution'], obj, rtol=1e-15, atol=1e-15)
    po, lens = f.flat('place_ones')
    assert np.array_equal(lens, f['ones'])
    pm, lm = f.flat('place_multi')
    cm, _ = f.flat('count_multi')
    assert np.array_equal(lm, f['multi']) and np.all(cm > 1)
    assert po.min() >= 0 and po.max() < 61 * 61
    per_frame = (f['ones'].sum() + cm.sum()) / n
    # every frame is normalised to mean_count before rotation; the rotation
    # drops the corners' share, so the mean lies a little below 2000
    assert 1600 < per_frame <= 2000 * 1.02
    # the same seeded configuration writes the same file
    gen2 = DataGenerator(cfg)
    out2 = gen2.make_data()
    assert np.array_equal(out2['place_ones'], po) and np.array_equal(out2['count_multi'], cm)
    # EMC reads it
    from dset import Dataset
    ds = Dataset(str(tmp_path / 'photons.h5'), 61 * 61, need_scaling=True)
    assert ds.num_data == n


def test_datagenerator_hetero_background_and_parse(tmp_path):
    from make_data import DataGenerator
    from rspi.photonfile import PhotonsFile
    cfg = _config(str(tmp_path / 'sim.ini'), size=61, n=64, kind='mix', hetro=True,
                  random=True, bg=50., out='p.npz')
    gen = DataGenerator(cfg)
    gen.make_obj()
    out = gen.make_data()
    f = PhotonsFile(str(tmp_path / 'p.npz'))
    assert 'rigid' in f and 'wobble' in f and 'true_wobbles' in f
    assert f['true_wobbles'].shape == (64, 2)
    assert f['bg'].shape == (61, 61)
    assert out['ones'].shape == (64,)
    # parse_obj with bg rescales the stored background to bg_count photons
    gen2 = DataGenerator(cfg)
    gen2.parse_obj(bg=True)
    assert abs(gen2.bgmask_sum - 2 * 50.) < 1e-9
    with pytest.raises(KeyError):
        gen2.parse_obj()      # the reference reads 'solution', absent for a hetero object


def test_datagenerator_rejects_wobble_types_without_hetero(tmp_path):
    from make_data import DataGenerator
    cfg = _config(str(tmp_path / 'sim.ini'), n=4, kind='blur', hetro=False)
    gen = DataGenerator(cfg)
    with pytest.raises(ValueError):
        gen.make_data()


def test_datagenerator_without_frames(tmp_path):
    """num_data = 0 writes the object and empty frame datasets."""
    from make_data import DataGenerator
    from rspi.photonfile import PhotonsFile
    cfg = _config(str(tmp_path / 'sim.ini'), n=0)
    gen = DataGenerator(cfg)
    out = gen.make_data()
    assert out['ones'].shape == (0,) and out['place_ones'].shape == (0,)
    f = PhotonsFile(str(tmp_path / 'photons.h5'))
    assert f['true_angles'].shape == (0,) and 'solution' in f
