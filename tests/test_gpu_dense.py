"""Dense-frame likelihood on the tensor cores (row a7 for frames stored as
dense uint16 counts): the BF16 digit matrices, the hi/lo split of the
rotated log-slices and the tcgen05 GEMM against FP64 references.

Tolerance of the GEMM: the products are exact (8-bit digits times 8-bit
BF16 mantissas) and the accumulation is FP32, so the result is compared with
the FP64 dot product of the same BF16 operands within
1e-5 * sum |K * (hi + lo)| + 1e-6 * |init * scale|."""
import numpy as np
import pytest
import torch

from oracle import emc_oracle as E

pytestmark = pytest.mark.gpu


def _call(name, *args):
    from rspi.lib import call
    call(name, *args)


def _p(t):
    from rspi.device import ptr
    return ptr(t)


def _s():
    from rspi.device import cur_stream
    return cur_stream()


def _gemm_case(n_frames, k_pad, n_brows, row_begin, row_end, num_rot, kmax, seed):
    rng = np.random.default_rng(seed)
    dev = torch.device('cuda')
    k = rng.integers(0, kmax + 1, (n_frames, k_pad))
    k[:, k_pad - 7:] = 0                                      # padding columns
    a0 = torch.from_numpy((k & 255).astype(np.float32)).to(dev, torch.bfloat16)
    a1 = None
    if kmax > 255:
        a1 = torch.from_numpy((k - (k & 255)).astype(np.float32)).to(dev, torch.bfloat16)
    lsl = rng.normal(0., 3., (n_brows, k_pad))
    lsl[:, :5] = -1000.                                       # out-of-detector sentinel
    t = torch.from_numpy(lsl)
    hi = t.to(torch.bfloat16)
    lo = (t - hi.double()).to(torch.bfloat16)
    n_states0 = (row_end + num_rot - 1) // num_rot + 1
    init = torch.from_numpy(rng.normal(-50., 10., n_states0)).to(dev)
    scales = torch.from_numpy(rng.lognormal(0., 0.3, n_frames)).to(dev)
    ld = n_frames + 3
    prob = torch.full((row_end - row_begin, ld), np.nan, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    hi_d, lo_d = hi.to(dev).contiguous(), lo.to(dev).contiguous()
    _call('rspi_dense_loglike', _p(a0), _p(a1), _p(hi_d), _p(lo_d), k_pad, n_frames, n_brows,
          num_rot, row_begin, row_end, _p(init), _p(scales), _p(prob), ld, _p(err), _s())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    # FP64 reference on the same BF16 operands
    kk = torch.from_numpy(k.astype(np.float64))
    lt = hi.double() + lo.double()                            # (n_brows, k_pad)
    rows = torch.arange(row_begin, row_end)
    dot = kk @ lt[:row_end - row_begin].T                    # (n_frames, rows)
    mag = kk @ lt[:row_end - row_begin].abs().T
    base = (init.cpu()[rows // num_rot][None, :] * scales.cpu()[:, None])
    want = (base + dot).T.numpy()
    tol = (1e-5 * mag + 1e-6 * base.abs()).T.numpy()
    got = prob.cpu().numpy()
    assert np.all(np.isnan(got[:, n_frames:]))               # beyond n_frames: untouched
    diff = np.abs(got[:, :n_frames].astype(np.float64) - want)
    assert np.all(diff <= tol), float((diff / tol).max())
    return diff


@pytest.mark.parametrize('n_frames,k_pad,n_brows,row_begin,row_end,kmax', [
    (128, 64, 128, 0, 128, 255),        # one tile, one k-block
    (300, 320, 260, 37, 237, 200),      # partial tiles, the stage ring wraps
    (200, 448, 150, 0, 150, 3000),      # two count digits
])
def test_dense_gemm_matches_fp64(n_frames, k_pad, n_brows, row_begin, row_end, kmax):
    # b rows of the buffer are rows row_begin.. of the likelihood matrix
    _gemm_case(n_frames, k_pad, n_brows, row_begin, row_end, num_rot=7, kmax=kmax, seed=k_pad)


def test_dense_frames_digits_exact():
    from rspi import geometry
    rng = np.random.default_rng(3)
    size = 33
    _, pm = E.generate_masks(size)
    sel, _, _ = geometry.sel_pixels(pm)
    k_pad = (sel.size + 63) // 64 * 64
    frames = rng.integers(0, 700, (9, size * size)).astype(np.uint16)
    frames[2] = 65535
    dev = torch.device('cuda')
    fr = torch.from_numpy(frames.view(np.int16)).to(dev)
    sel_t = torch.from_numpy(sel.astype('i4')).to(dev)
    a0 = torch.empty((9, k_pad), dtype=torch.bfloat16, device=dev)
    a1 = torch.empty((9, k_pad), dtype=torch.bfloat16, device=dev)
    kmax = torch.zeros(1, dtype=torch.int32, device=dev)
    _call('rspi_dense_frames', _p(fr), 9, size * size, _p(sel_t), sel.size, k_pad, _p(a0), _p(a1),
          _p(kmax), _s())
    torch.cuda.synchronize()
    want = np.zeros((9, k_pad), dtype=np.int64)
    want[:, :sel.size] = frames[:, sel]
    assert int(kmax.item()) == want.max() == 65535
    got = a0.double().cpu().numpy() + a1.double().cpu().numpy()
    assert np.array_equal(got, want)
    assert np.all(a0.double().cpu().numpy() <= 255)


def test_rot_log_split_matches_oracle():
    """hi + lo reproduces the FP64 oracle's rotated log-slices to 2^-16."""
    from helpers import golden_dataset, golden_states, load_golden
    from rspi import geometry
    from rspi.device import DevicePhotons, EStep
    g = load_golden('case_b')
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    _, pm = E.generate_masks(size)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']))
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='fp64')
    model = torch.from_numpy(g['model_in_1']).cuda()
    es.slices(model)
    sel, _, _ = geometry.sel_pixels(pm)
    k_pad = (sel.size + 63) // 64 * 64
    n_rows = es.n_rows
    hi = torch.empty((n_rows, k_pad), dtype=torch.bfloat16, device='cuda')
    lo = torch.empty_like(hi)
    amax = torch.zeros(1, dtype=torch.float32, device='cuda')
    _call('rspi_rot_log_split', _p(es.holo), es.n_states0, num_rot, _p(es.rot_cs), size, _p(es.bg),
          _p(es.sel_pix), es.n_sel, k_pad, 0, n_rows, _p(hi), _p(lo), _p(amax), _s())
    torch.cuda.synchronize()
    got = (hi.double() + lo.double()).cpu().numpy()
    want = np.zeros_like(got)
    for s in range(sx.size):
        want[s * num_rot:(s + 1) * num_rot, :sel.size] = E.log_slices_for_state(
            g['model_in_1'], sx[s], sy[s], dia[s], size, ds['bg'], num_rot, pm < 1)
    assert np.all(np.abs(got - want) <= 2. ** -16 * np.abs(want) + 1e-12)
    assert np.all(got[:, sel.size:] == 0)
    np.testing.assert_allclose(float(amax.item()), np.abs(want).max(), rtol=1e-6)


def _dense_from_sparse(ds):
    n, npix = ds['num_data'], ds['num_pix']
    frames = np.zeros((n, npix), dtype=np.int64)
    kmat = E.sparse_frames(ds).toarray()
    frames[:] = kmat
    return frames.astype(np.uint16)


@pytest.mark.parametrize('gemm', ['i8', 'bf16'])
@pytest.mark.parametrize('name', ['case_a', 'case_b'])
def test_dense_estep_matches_oracle(name, gemm):
    """form='dense': the GEMM likelihoods within the FP32 bound of the FP64
    oracle, and after FP64 rescoring the same argmax, maximum and
    log-sum-exp as the oracle."""
    from helpers import golden_dataset, golden_states, load_golden
    from rspi.device import DevicePhotons, EStep
    g = load_golden(name)
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    _, pm = E.generate_masks(size)
    frames = _dense_from_sparse(ds)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']), frames=frames)
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='dense',
               slice_budget_bytes=1 << 16, dense_gemm=gemm)
    assert es.dense_gemm == gemm
    assert es.chunk_rows < es.n_rows or es.n_rows <= 128      # chunks when there are several tiles
    model = torch.from_numpy(g['model_in_1']).cuda()
    es.run(model)
    torch.cuda.synchronize()
    want, _, _ = E.calc_prob(g['model_in_1'], ds, sx, sy, dia, size, num_rot, pm,
                             E.get_scales(ds, bool(g['need_scaling'])))
    got = es.frame_prob().cpu().numpy().astype(np.float64)
    kmat = E.sparse_frames(ds, pm < 1)
    lsl = np.concatenate([E.log_slices_for_state(g['model_in_1'], sx[s], sy[s], dia[s], size,
                                                 ds['bg'], num_rot, pm < 1) for s in range(sx.size)])
    mag = np.asarray(abs(kmat) @ np.abs(lsl).T).T                # sum |K L| per (row, frame)
    if gemm == 'i8':
        # quantisation 2^-22 per photon, then the FP32 store
        phot = np.asarray(kmat.sum(1)).ravel()[None, :]
        tol = 2. ** -22 * phot + 2. ** -23 * np.abs(want) + 1e-9
    else:
        tol = 2. ** -16 * mag + 1e-5 * mag + 1e-6 * np.abs(want)
    assert np.all(np.abs(got - want) <= tol)
    print('dense (%s) LL max rel err vs FP64: %.3e' %
          (gemm, float((np.abs(got - want) / np.maximum(np.abs(want), 1)).max())))
    maxll, rmax, logz = es.reduce()
    torch.cuda.synchronize()
    mx, am = E.get_rmax(want)
    assert np.array_equal(rmax.cpu().numpy(), am)
    np.testing.assert_allclose(maxll.cpu().numpy(), mx, rtol=1e-11)
    lz, _ = E.posterior(want)
    np.testing.assert_allclose(logz.cpu().numpy(), lz, rtol=1e-11)


def test_emc_dense_form_matches_reference(tmp_path):
    """EMC with form = dense on a photons file holding dense frames: two
    iterations reproduce the reference goldens (argmax and model)."""
    from emc import EMC
    from helpers import golden_dataset, load_golden, write_case
    from rspi.photonfile import write_photons
    g = load_golden('case_a')
    cfg = write_case(str(tmp_path), g, extra='form = dense\n')
    ds = golden_dataset(g)
    size = int(g['size'])
    out = dict(num_pix=np.array([size * size]), ones=g['ones'], multi=g['multi'],
               place_ones=g['place_ones'], place_multi=g['place_multi'],
               count_multi=g['count_multi'], frames=_dense_from_sparse(ds))
    if 'bg' in g:
        out['bg'] = g['bg']
    write_photons(str(tmp_path / 'photons.npz'), out)
    rec = EMC(cfg)
    assert rec.estep.form == 'dense'
    rec.model = g['model_in_1'].copy()
    for it in (1, 2):     # the golden chain: model_in_2 is model_out_1
        rec.run_iteration(None)
        assert np.array_equal(rec.rmax, g['rmax_%d' % it])
        np.testing.assert_allclose(rec.model, g['model_out_%d' % it], rtol=1e-9, atol=1e-12)


def test_dense_estep_large_detector_global_rescore_rows():
    """A 215-pixel detector: the FP64 rescoring row (about 36,000 likelihood
    pixels) exceeds shared memory and is built in global scratch; argmax,
    maximum and log-sum-exp still equal the oracle's."""
    from helpers import random_photons
    from rspi.device import DevicePhotons, EStep
    size, n, num_rot = 215, 12, 4
    d = random_photons(size, n, 3000., 21)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, True)
    sx, sy, dia, _ = E.generate_states(E.parse_triple('0 1 2'), E.parse_triple('0 0 1'),
                                       E.parse_triple('6 8 2'))
    _, pm = E.generate_masks(size)
    rng = np.random.default_rng(2)
    model = rng.random(size * size) + 1j * rng.random(size * size)
    frames = _dense_from_sparse(ds)
    ph = DevicePhotons(d['ones'], d['multi'], d['place_ones'], d['place_multi'], d['count_multi'],
                       size * size, True, frames=frames)
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='dense')
    assert es.row_scratch is not None
    es.run(torch.from_numpy(model).cuda())
    maxll, rmax, logz = es.reduce()
    torch.cuda.synchronize()
    want, _, _ = E.calc_prob(model, ds, sx, sy, dia, size, num_rot, pm, E.get_scales(ds, True))
    mx, am = E.get_rmax(want)
    assert np.array_equal(rmax.cpu().numpy(), am)
    np.testing.assert_allclose(maxll.cpu().numpy(), mx, rtol=1e-11)
    lz, _ = E.posterior(want)
    np.testing.assert_allclose(logz.cpu().numpy(), lz, rtol=1e-11)


def test_dense_i8_gemm_exact():
    """The integer GEMM equals init * scale + 2^-21 sum K Lq computed
    exactly (int64), up to the FP32 store; partial tiles, a wrapping stage
    ring and negative digits (the -1000 sentinel) included."""
    rng = np.random.default_rng(8)
    n_frames, k_pad, n_brows, row_begin, row_end, num_rot = 300, 384, 260, 37, 237, 7
    dev = torch.device('cuda')
    k = rng.integers(0, 256, (n_frames, k_pad))
    k[:, k_pad - 9:] = 0
    lq = rng.integers(-(1000 << 21), 60 << 21, (n_brows, k_pad)).astype(np.int64)
    planes = np.stack([(lq >> (8 * j)) & 255 for j in range(4)]).astype(np.uint8)
    a = torch.from_numpy(k.astype(np.uint8)).to(dev)
    dg = torch.from_numpy(planes).to(dev).contiguous()
    n_states0 = (row_end + num_rot - 1) // num_rot + 1
    init = torch.from_numpy(rng.normal(-50., 10., n_states0)).to(dev)
    scales = torch.from_numpy(rng.lognormal(0., 0.3, n_frames)).to(dev)
    prob = torch.full((row_end - row_begin, n_frames), np.nan, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _call('rspi_dense_loglike_i8', _p(a), _p(dg), k_pad, n_frames, n_brows, num_rot, row_begin,
          row_end, _p(init), _p(scales), _p(prob), n_frames, _p(err), _s())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    exact = k.astype(np.int64) @ lq[:row_end - row_begin].T          # (frames, rows), int64
    rows = np.arange(row_begin, row_end)
    base = init.cpu().numpy()[rows // num_rot][None, :] * scales.cpu().numpy()[:, None]
    want = (base + exact * 2. ** -21).T
    got = prob.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(got - want) <= 2. ** -23 * np.abs(want) + 1e-6)


def test_rot_log_fixed_matches_oracle():
    """The four digit planes rebuild rint(L 2^21) of the oracle's rotated
    log-slices (|error| <= 2^-22)."""
    from helpers import golden_dataset, golden_states, load_golden
    from rspi import geometry
    from rspi.device import DevicePhotons, EStep
    g = load_golden('case_a')
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    _, pm = E.generate_masks(size)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']))
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='fp64')
    es.slices(torch.from_numpy(g['model_in_1']).cuda())
    sel, _, _ = geometry.sel_pixels(pm)
    k_pad = (sel.size + 127) // 128 * 128
    n_rows = es.n_rows
    dg = torch.empty((4, n_rows, k_pad), dtype=torch.uint8, device='cuda')
    err = torch.zeros(1, dtype=torch.int32, device='cuda')
    _call('rspi_rot_log_fixed', _p(es.holo), es.n_states0, num_rot, _p(es.rot_cs), size, _p(es.bg),
          _p(es.sel_pix), es.n_sel, k_pad, 0, n_rows, n_rows, _p(dg), _p(err), _s())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    p = dg.cpu().numpy().astype(np.int64)
    lq = p[0] + (p[1] << 8) + (p[2] << 16) + (p[3].astype(np.int8).astype(np.int64) << 24)
    got = lq * 2. ** -21
    want = np.zeros_like(got)
    for s in range(sx.size):
        want[s * num_rot:(s + 1) * num_rot, :sel.size] = E.log_slices_for_state(
            g['model_in_1'], sx[s], sy[s], dia[s], size, ds['bg'], num_rot, pm < 1)
    assert np.all(np.abs(got - want) <= 2. ** -22 + 1e-12 * np.abs(want))


def test_dense_frames_u8():
    from rspi import geometry
    rng = np.random.default_rng(5)
    size = 29
    _, pm = E.generate_masks(size)
    sel, _, _ = geometry.sel_pixels(pm)
    k_pad = (sel.size + 127) // 128 * 128
    frames = rng.integers(0, 256, (7, size * size)).astype(np.uint16)
    fr = torch.from_numpy(frames.view(np.int16)).cuda()
    a = torch.empty((7, k_pad), dtype=torch.uint8, device='cuda')
    kmax = torch.zeros(1, dtype=torch.int32, device='cuda')
    sel_t = torch.from_numpy(sel.astype('i4')).cuda()
    _call('rspi_dense_frames_u8', _p(fr), 7, size * size, _p(sel_t), sel.size, k_pad, _p(a),
          _p(kmax), _s())
    torch.cuda.synchronize()
    want = np.zeros((7, k_pad), dtype=np.int64)
    want[:, :sel.size] = frames[:, sel]
    assert np.array_equal(a.cpu().numpy().astype(np.int64), want)
    assert int(kmax.item()) == want.max()
