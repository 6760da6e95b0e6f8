"""E-step parity on the GPU (rows a1-a9): librspi vs the pinned FP64 oracle
and the reference goldens.  Integer results (prefix sums, counts, powder,
entry lists, argmax) are compared bit-exactly; floating point within the
stated tolerances."""
import numpy as np
import pytest
import torch

from helpers import GOLDEN_CASES, golden_dataset, golden_states, load_golden, random_photons
from oracle import emc_oracle as E

pytestmark = pytest.mark.gpu

# FP64 pipeline vs FP64 oracle: only summation order differs
RTOL_F64 = 1e-11
# FP32 slices (FP64 accumulation): the 1e-5 bound on the likelihood
RTOL_F32 = 1e-5


def _photons(ds, need_scaling):
    from rspi.device import DevicePhotons
    return DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                         ds['count_multi'], ds['num_pix'], need_scaling)


def _estep(ph, size, num_rot, sx, sy, dia, bg, **kw):
    from rspi.device import EStep
    _, pm = E.generate_masks(size)
    return EStep(ph, size, num_rot, sx, sy, dia, pm, bg, **kw)


def _cases():
    out = []
    for name in GOLDEN_CASES:
        g = load_golden(name)
        out.append((name, golden_dataset(g), bool(g['need_scaling'])))
    for size, n, seed, kw in ((17, 1, 1, {}), (37, 33, 2, dict(empty_frames=(0, 5), masked_frames=(7,))),
                              (25, 40, 3, dict(heavy=3))):
        d = random_photons(size, n, 30. * size, seed, **kw)
        ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                             d['count_multi'], size * size, True)
        out.append(('rand%d' % size, ds, True))
    return out


CASES = _cases()


@pytest.mark.parametrize('name,ds,need_scaling', CASES, ids=[c[0] for c in CASES])
def test_photon_setup_bit_exact(name, ds, need_scaling):
    ph = _photons(ds, need_scaling)
    assert np.array_equal(ph.ones_accum.cpu().numpy(), ds['ones_accum'])
    assert np.array_equal(ph.multi_accum.cpu().numpy(), ds['multi_accum'])
    assert ph.mean_count == ds['mean_count']
    if need_scaling:
        assert np.array_equal(ph.counts.cpu().numpy(), ds['counts'])
    assert np.array_equal(ph.scales.cpu().numpy(), E.get_scales(ds, need_scaling))
    assert np.array_equal(ph.powder.cpu().numpy(), E.get_powder(ds))


@pytest.mark.parametrize('name,ds,need_scaling', CASES, ids=[c[0] for c in CASES])
def test_ll_entry_lists_bit_exact(name, ds, need_scaling):
    from rspi import geometry
    size = int(round(np.sqrt(ds['num_pix'])))
    ph = _photons(ds, need_scaling)
    _, pm = E.generate_masks(size)
    sel, pix2sel, p_pad = geometry.sel_pixels(pm)
    ll = ph.ll_entries(torch.from_numpy(pix2sel).cuda(), p_pad)
    ent = ll['entries'].cpu().numpy().view(np.uint32).reshape(-1, 32)
    off = ll['row_off'].cpu().numpy()
    kmat = E.sparse_frames(ds, pm < 1)
    for d in range(ds['num_data']):
        rows = ent[off[d]:off[d + 1]]
        c = (rows >> 16).astype(np.int64)
        k = (rows & 0xffff).astype(np.int64)
        lanes = np.broadcast_to(np.arange(32), rows.shape)
        assert np.all(c % 32 == lanes)               # bank-conflict-free layout
        got = np.zeros(sel.size + 32, dtype=np.int64)
        np.add.at(got, c[k > 0], k[k > 0])
        want = np.zeros(sel.size + 32, dtype=np.int64)
        row = kmat.getrow(d)
        want[row.indices] = row.data.astype(np.int64)
        assert np.array_equal(got, want), d
    order = ll['order'].cpu().numpy()
    rows = ll['frame_rows'].cpu().numpy()
    assert np.all(np.diff(rows[order]) <= 0)


def frame_photons16(es):
    """Each frame's sorted likelihood-column indices, one per photon (counts
    expanded), read from the 16-bit entry rows of ``es``."""
    l16 = es.ll16
    ent = l16['entries'].cpu().numpy().view(np.uint16).astype(np.int64)
    off = l16['row_off'].cpu().numpy()
    pz = es.p_row - 32
    out = []
    for d in range(off.size - 1):
        rows = [ent[(r >> 1) * 64 + 2 * np.arange(32) + (r & 1)] for r in range(off[d], off[d + 1])]
        v = np.concatenate(rows) if rows else np.zeros(0, np.int64)
        out.append(np.sort(v[v < pz]))
    return out


def _golden_estep(g, **kw):
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    ph = _photons(ds, bool(g['need_scaling']))
    return ds, _estep(ph, size, num_rot, sx, sy, dia, ds['bg'], **kw)


@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_holo_msum_vscale(name):
    g = load_golden(name)
    ds, es = _golden_estep(g)
    size = int(g['size'])
    sx, sy, dia, _ = golden_states(g)
    model = torch.from_numpy(g['model0']).cuda()
    es.slices(model)
    holo = es.holo.cpu().numpy()
    np.testing.assert_allclose(holo[:g['holo'].shape[0]], g['holo'], rtol=1e-13)
    _, pm = E.generate_masks(size)
    msums, vscale = E.msum_vscale(g['model0'], sx, sy, dia, size, ds['bg'], pm, E.get_powder(ds))
    np.testing.assert_allclose(es.msum.cpu().numpy(), msums, rtol=1e-13)
    np.testing.assert_allclose(float(es.vscale), vscale, rtol=1e-13)


@pytest.mark.parametrize('name', GOLDEN_CASES)
@pytest.mark.parametrize('form', ['fp64', 'screen'])
def test_rotated_log_slices(name, form):
    """Row-major rotated log-slices (the slice layout of the streaming
    kernels; the frame-set layout holds the same values, checked by
    test_sets_slice_layout_bit_identical) against the oracle."""
    g = load_golden(name)
    ds, es = _golden_estep(g, form=form, kernel='stream')
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    es.slices(torch.from_numpy(g['model0']).cuda())
    es.rot_slices(0, es.chunk_rows)
    lsl = es.lsl.double().cpu().numpy()
    _, pm = E.generate_masks(size)
    sel = pm < 1
    for r in range(min(es.chunk_rows, 3 * num_rot)):
        s0, j = divmod(r, num_rot)
        w = E.holo_slice(g['model0'], sx[s0], sy[s0], dia[s0], 1., 1., size, ds['bg'])
        want = E.rotate_slice(w, j * np.pi / num_rot, 1., size, ds['bg'], 1)[sel]
        got = lsl[r, :sel.sum()]
        if form == 'fp64':
            np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13)
        else:
            np.testing.assert_allclose(got, want.astype(np.float32), rtol=1e-6, atol=1e-6)
        assert np.all(lsl[r, sel.sum():] == 0)


@pytest.mark.parametrize('name', GOLDEN_CASES)
@pytest.mark.parametrize('it', [1, 2])
def test_loglike_fp64_matches_reference(name, it):
    g = load_golden(name)
    _, es = _golden_estep(g)
    es.run(torch.from_numpy(g['model_in_%d' % it]).cuda())
    prob = es.frame_prob().cpu().numpy()
    np.testing.assert_allclose(prob, g['prob_%d' % it], rtol=RTOL_F64, atol=0)
    maxll, rmax, logz = es.reduce()
    assert np.array_equal(rmax.cpu().numpy(), g['rmax_%d' % it])
    np.testing.assert_allclose(maxll.cpu().numpy(), g['prob_%d' % it].max(0), rtol=RTOL_F64)
    want_logz, _ = E.posterior(g['prob_%d' % it])
    np.testing.assert_allclose(logz.cpu().numpy(), want_logz, rtol=RTOL_F64)


@pytest.mark.parametrize('name', GOLDEN_CASES)
@pytest.mark.parametrize('it', [1, 2])
def test_screened_form_matches_fp64(name, it):
    """FP32 screening + FP64 rescoring: the FP32 matrix is within 1e-5 of
    FP64 everywhere, and rmax/max/logz equal the FP64 form's."""
    g = load_golden(name)
    _, es = _golden_estep(g, form='screen')
    _, ref = _golden_estep(g, form='fp64')
    model = torch.from_numpy(g['model_in_%d' % it]).cuda()
    es.run(model)
    ref.run(model)
    screened = es.frame_prob().cpu().numpy().astype(np.float64)
    want = g['prob_%d' % it]
    assert (np.abs(screened - want) / np.abs(want)).max() <= RTOL_F32
    maxll, rmax, logz = es.reduce()
    rmax64 = ref.reduce()[1].cpu().numpy()
    assert np.array_equal(rmax.cpu().numpy(), g['rmax_%d' % it])
    assert np.array_equal(rmax.cpu().numpy(), rmax64)
    np.testing.assert_allclose(maxll.cpu().numpy(), ref.maxll.cpu().numpy(), rtol=1e-15)
    np.testing.assert_allclose(logz.cpu().numpy(), ref.logz.cpu().numpy(), rtol=1e-13)
    want_logz, _ = E.posterior(want)
    np.testing.assert_allclose(logz.cpu().numpy(), want_logz, rtol=RTOL_F64)
    assert es.n_candidates >= g['prob_%d' % it].shape[1]


def test_screen_candidates_cover_posterior_mass():
    """Every state with posterior above exp(-delta) is rescored, and the
    capacity grows when a frame has more candidates than reserved."""
    g = load_golden('case_b')
    _, es = _golden_estep(g, form='screen', delta=200., cand_per_frame=1)
    es.run(torch.from_numpy(g['model_in_1']).cuda())
    es.reduce()
    want = g['prob_1']
    off = es.cand_off.cpu().numpy()
    cd = es.cand_d.cpu().numpy()[:off[-1]]
    cr = es.cand_r.cpu().numpy()[:off[-1]]
    cl = es.cand_ll.cpu().numpy()[:off[-1]]
    assert es.capacity >= off[-1] > 1024
    keep = want >= want.max(0) - 200.
    got = np.zeros_like(keep)
    got[cr, cd] = True
    assert np.all(got[keep])
    np.testing.assert_allclose(cl, want[cr, cd], rtol=RTOL_F64)


@pytest.mark.parametrize('form,kernel', [('fp64', 'stream'), ('fp64', 'dynamic'),
                                         ('screen', 'stream')])
@pytest.mark.parametrize('tile,warps', [(1, 1), (2, 4), (3, 32), (1, 7), (8, 16), (4, 32)])
def test_tiling_does_not_change_results(tile, warps, form, kernel):
    g = load_golden('case_a')
    _, ref = _golden_estep(g, form=form, kernel=kernel)
    ref.run(torch.from_numpy(g['model_in_1']).cuda())
    _, es = _golden_estep(g, states_per_tile=tile, warps=warps, form=form, kernel=kernel)
    es.run(torch.from_numpy(g['model_in_1']).cuda())
    rtol = 1e-14 if form == 'fp64' else 1e-6
    np.testing.assert_allclose(es.frame_prob().cpu().numpy(), ref.frame_prob().cpu().numpy(), rtol=rtol)


def test_kernel_choice_is_checked():
    g = load_golden('case_a')
    for form, kernel in (('screen', 'dynamic'), ('fp64', 'quad4'), ('screen', 'wide')):
        with pytest.raises(ValueError):
            _golden_estep(g, form=form, kernel=kernel)


@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_stream_kernel_bit_identical_to_dynamic(name):
    """The FP64 streaming kernel keeps the per-lane order and the warp
    reduction of the dynamic kernel, so the likelihoods are bit-identical."""
    g = load_golden(name)
    _, a = _golden_estep(g, kernel='dynamic')
    _, b = _golden_estep(g, kernel='stream', warps=3)
    m = torch.from_numpy(g['model_in_2']).cuda()
    a.run(m)
    b.run(m)
    assert torch.equal(a.frame_prob(), b.frame_prob())


def test_chunked_slices_match_single_pass():
    g = load_golden('case_b')
    _, ref = _golden_estep(g)
    ref.run(torch.from_numpy(g['model_in_1']).cuda())
    _, es = _golden_estep(g, states_per_tile=2, slice_budget_bytes=7 * 32 * 8 * 2)
    assert es.chunk_rows < es.n_rows
    es.run(torch.from_numpy(g['model_in_1']).cuda())
    np.testing.assert_allclose(es.frame_prob().cpu().numpy(), ref.frame_prob().cpu().numpy(), rtol=1e-14)


@pytest.mark.parametrize('form', ['fp64', 'screen'])
@pytest.mark.parametrize('size,n,seed,kw', [
    (17, 1, 1, {}),
    (37, 33, 2, dict(empty_frames=(0, 5), masked_frames=(7,))),
    (25, 40, 3, dict(heavy=3)),
    (5, 3, 4, {}),        # no likelihood pixels at all: vscale = 0/0 as in the reference
])
def test_random_shapes_vs_oracle(size, n, seed, kw, form):
    d = random_photons(size, n, 30. * size, seed, **kw)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, True)
    sx, sy, dia, _ = E.generate_states((-1., 1., 2), (0., 1., 2), (2., 3., 2))
    num_rot = 5
    ph = _photons(ds, True)
    es = _estep(ph, size, num_rot, sx, sy, dia, ds['bg'], form=form)
    model = np.random.default_rng(seed).random(size * size) + 1j * np.random.default_rng(seed + 1).random(size * size)
    es.run(torch.from_numpy(model).cuda())
    _, pm = E.generate_masks(size)
    with np.errstate(invalid='ignore', divide='ignore'):
        want, _, _ = E.calc_prob(model, ds, sx, sy, dia, size, num_rot, pm, E.get_scales(ds, True))
    got = es.frame_prob().cpu().numpy().astype(np.float64)
    if np.isnan(want).all():
        assert np.isnan(got).all()
    else:
        np.testing.assert_allclose(got, want, rtol=RTOL_F64 if form == 'fp64' else RTOL_F32,
                                   atol=1e-9)
    _, rmax, _ = es.reduce()
    _, want_rmax = E.get_rmax(want)
    assert np.array_equal(rmax.cpu().numpy(), want_rmax)


@pytest.mark.parametrize('kernel', ['stream', 'quad4'])
@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_screen_kernels_match_reference(name, kernel):
    g = load_golden(name)
    _, es = _golden_estep(g, form='screen', kernel=kernel)
    for it in (1, 2):
        es.run(torch.from_numpy(g['model_in_%d' % it]).cuda())
        screened = es.frame_prob().cpu().numpy().astype(np.float64)
        want = g['prob_%d' % it]
        assert (np.abs(screened - want) / np.abs(want)).max() <= RTOL_F32
        _, rmax, _ = es.reduce()
        assert np.array_equal(rmax.cpu().numpy(), g['rmax_%d' % it])


@pytest.mark.parametrize('parts,warps', [(None, 32), (2, 24), (3, 7), (4, 32)])
@pytest.mark.parametrize('name,ds,need_scaling', CASES, ids=[c[0] for c in CASES])
def test_quad4_kernel_matches_stream_kernel(name, ds, need_scaling, parts, warps):
    """The four-row frame-quad kernel (column parts staged one after
    another, running sums per frame slot between parts) gives the
    interleaved kernel's FP32 likelihoods within 1e-6 of the largest term,
    and the same FP64-rescored argmax / maximum / log-sum-exp, on every case
    (empty, heavy and single-frame data included)."""
    size = int(round(np.sqrt(ds['num_pix'])))
    num_rot = 5
    sx, sy, dia, _ = E.generate_states(E.parse_triple('-1 1 3'), E.parse_triple('0 0 1'),
                                       E.parse_triple('2 3 2'))
    rng = np.random.default_rng(size)
    model = torch.from_numpy(rng.random(size * size) + 1j * rng.random(size * size)).cuda()
    out = {}
    for kernel, tile, kw in (('stream', 2, {}), ('quad4', 4, dict(screen_parts=parts))):
        ph = _photons(ds, need_scaling)
        es = _estep(ph, size, num_rot, sx, sy, dia, ds['bg'], form='screen', kernel=kernel,
                    states_per_tile=tile, warps=warps, **kw)
        es.run(model)
        maxll, rmax, logz = es.reduce()
        torch.cuda.synchronize()
        out[kernel] = (es.frame_prob().cpu().numpy().astype(np.float64), maxll.cpu().numpy(),
                       rmax.cpu().numpy(), logz.cpu().numpy())
        if kernel == 'quad4':
            assert es.wide['n_parts'] == (parts or 1)
    a, b = out['stream'], out['quad4']
    scale = np.abs(a[0]).max(0, keepdims=True) + 1.
    assert np.all(np.abs(a[0] - b[0]) <= 1e-6 * scale)
    assert np.array_equal(a[2], b[2])
    np.testing.assert_allclose(a[1], b[1], rtol=1e-14)
    np.testing.assert_allclose(a[3], b[3], rtol=1e-12)


@pytest.mark.parametrize('n,parts', [(61, 1), (300, 2), (45, 3)])
def test_quad4_layout_entries(n, parts):
    """Four-row frame quads: every frame's photons once per column part, in
    its eight lanes, lane j holding local columns = j (mod 8) as q = local / 8;
    the pad q = part_w / 8 (zero columns) elsewhere; group ranges part-major
    with each (quad, part) as long as its longest frame needs; frames taken
    within windows of consecutive frames."""
    from rspi.device import QUAD4_WINDOW
    size = 37
    d = random_photons(size, n, 40. * size, 14, empty_frames=(2, 9), heavy=5)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, False)
    sx, sy, dia, _ = E.generate_states(E.parse_triple('0 0 1'), E.parse_triple('0 0 1'),
                                       E.parse_triple('2 2 1'))
    es_q = _estep(_photons(ds, False), size, 3, sx, sy, dia, ds['bg'], form='screen',
                  kernel='quad4', states_per_tile=4, screen_parts=parts)
    torch.cuda.synchronize()
    w = es_q.wide
    pz = es_q.p_row - 32
    pw, nq = w['part_w'], w['n_pairs']
    assert w['n_parts'] == parts and pw % 8 == 0 and parts * pw >= pz
    q = w['entries'].cpu().numpy().view(np.uint16).reshape(-1, 32, 4).astype(np.int64)
    j = (np.arange(32) % 8)[None, :, None]
    local = q * 8 + j                                          # local column of each slot
    goff = w['group_off'].cpu().numpy()
    qf = w['pair_frames'].cpu().numpy()
    assert nq == (n + 3) // 4 and goff.size == parts * nq + 1 and np.all(np.diff(goff) >= 0)
    photons = frame_photons16(es_q)
    seen = []
    for qd in range(nq):
        for uu in range(4):
            f = qf[4 * qd + uu]
            got = []
            for h in range(parts):
                blk = local[goff[h * nq + qd]:goff[h * nq + qd + 1], 8 * uu:8 * uu + 8]
                real = blk < pw
                assert np.all(blk[~real] == pw + np.broadcast_to(np.arange(8)[None, :, None],
                                                                blk.shape)[~real])
                if f < 0:
                    assert not real.any()
                got.append(blk[real] + h * pw)
            if f < 0:
                continue
            seen.append(f)
            assert np.array_equal(np.sort(np.concatenate(got)), photons[f]), f
    assert sorted(seen) == list(range(n))
    assert np.all(qf[:n] // QUAD4_WINDOW == np.arange(n) // QUAD4_WINDOW)
    # each (quad, part) range is as long as its longest frame needs
    for h in range(parts):
        for qd in range(nq):
            fr = [f for f in qf[4 * qd:4 * qd + 4] if f >= 0]
            need = 0
            for f in fr:
                ref = photons[f]
                cols = ref[ref // pw == h] % pw
                if cols.size:
                    need = max(need, -(-np.bincount(cols % 8, minlength=8).max() // 4))
            assert goff[h * nq + qd + 1] - goff[h * nq + qd] == need


@pytest.mark.parametrize('dtype,code', [(torch.float32, 0), (torch.float64, 1)])
def test_paired_holo_slices_bit_identical(dtype, code):
    """rspi_rot_log_slices_pairs (two 16-byte loads per bilinear sample from
    the paired copy) gives the bits of rspi_rot_log_slices on row ranges
    that start and end inside a state's rotations, and the same abs_max."""
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    g = load_golden('case_b')
    _, es = _golden_estep(g, form='screen')
    es.slices(torch.from_numpy(g['model_in_1']).cuda())
    n = es.n_rows
    for r0, r1 in ((0, n), (3, n - 5), (es.num_rot + 1, min(n, 3 * es.num_rot + 2)), (7, 8)):
        outs = []
        for fn, src in (('rspi_rot_log_slices', es.holo), ('rspi_rot_log_slices_pairs',
                                                            es.holo_pairs)):
            out = torch.full((r1 - r0, es.p_row), 7., dtype=dtype, device='cuda')
            amax = torch.zeros(1, dtype=torch.float32, device='cuda')
            call(fn, ptr(src), es.n_states0, es.num_rot, ptr(es.rot_cs), es.size, ptr(es.bg),
                 ptr(es.sel_pix), es.n_sel, es.p_row, r0, r1, ptr(out), code, ptr(amax),
                 cur_stream())
            torch.cuda.synchronize()
            outs.append((out.cpu().numpy(), float(amax.item())))
        a, b = outs
        assert np.array_equal(a[0].view(np.uint8), b[0].view(np.uint8)), (r0, r1)
        assert a[1] == b[1] and a[1] > 0.


@pytest.mark.parametrize('set_order', ['grouped', 'rank'])
@pytest.mark.parametrize('parts,warps', [(None, 32), (2, 16), (3, 7), (4, 32)])
@pytest.mark.parametrize('name,ds,need_scaling', CASES, ids=[c[0] for c in CASES])
def test_sets_kernel_matches_stream_kernel(name, ds, need_scaling, parts, warps, set_order):
    """The frame-set kernel (column parts copied in by TMA one after another,
    one lane per frame, running sums per column between parts, the
    likelihood columns in set order) gives FP32 likelihoods within the
    screening bound eps_d of the FP64 form's (as the plain streaming kernel
    does; the two sum in different orders, so they differ from each other by
    rounding), and the same FP64-rescored argmax / maximum / log-sum-exp, on
    every case (empty, heavy and single-frame data included)."""
    size = int(round(np.sqrt(ds['num_pix'])))
    num_rot = 5
    sx, sy, dia, _ = E.generate_states(E.parse_triple('-1 1 3'), E.parse_triple('0 0 1'),
                                       E.parse_triple('2 3 2'))
    rng = np.random.default_rng(size)
    model = torch.from_numpy(rng.random(size * size) + 1j * rng.random(size * size)).cuda()
    ref = _estep(_photons(ds, need_scaling), size, num_rot, sx, sy, dia, ds['bg'], form='fp64')
    ref.run(model)
    ref.reduce()
    want = ref.frame_prob().cpu().numpy()
    out = {}
    for kernel, tile, kw in (('stream', 2, {}),
                             ('sets', 4, dict(screen_parts=parts, set_order=set_order))):
        ph = _photons(ds, need_scaling)
        es = _estep(ph, size, num_rot, sx, sy, dia, ds['bg'], form='screen', kernel=kernel,
                    states_per_tile=tile, warps=warps, **kw)
        es.run(model)
        maxll, rmax, logz = es.reduce()
        torch.cuda.synchronize()
        ph.err.check('sets kernel')
        got = es.frame_prob().cpu().numpy().astype(np.float64)
        out[kernel] = (got, maxll.cpu().numpy(), rmax.cpu().numpy(), logz.cpu().numpy())
        if kernel == 'sets':
            assert es.wide['n_parts'] == (parts or 1)
        # eps_d = 2^-24 ((rows_d + 8) photons_d lmax + |L|): the bound the
        # candidate threshold is built on, rows_d the kernel's summation length
        rows = np.diff(es._eps_rows().cpu().numpy()).astype(np.float64)
        phot = es.ll['frame_sel_photons'].cpu().numpy().astype(np.float64)
        lmax = float(es.lmax.cpu().numpy().reshape(-1)[0])
        eps = 2. ** -24 * ((rows + 8.) * phot * lmax + np.abs(want) + 1.)
        fin = np.isfinite(want)
        assert np.array_equal(fin, np.isfinite(got))
        err = np.where(fin, np.abs(got - want), 0.)
        worst = np.unravel_index(np.argmax(err / np.where(fin, eps, 1.)), err.shape)
        assert np.all(err <= np.where(fin, eps, 0.)), (kernel, worst, err[worst], eps[worst],
                                                        want[worst])
    a, b = out['stream'], out['sets']
    assert np.array_equal(a[2], b[2])
    np.testing.assert_allclose(a[1], b[1], rtol=1e-14)
    np.testing.assert_allclose(a[3], b[3], rtol=1e-12)


@pytest.mark.parametrize('set_order', ['grouped', 'rank'])
@pytest.mark.parametrize('n,parts', [(61, 1), (300, 2), (45, 3), (33, 4)])
def test_sets_layout_entries(n, parts, set_order):
    """Frame sets: every frame's photons of each column part once, in its own
    lane, within its quarter warp's first D_q steps, D_q the fewest any
    schedule needs (its largest frame or class total), in which the eight
    lanes read eight distinct bank classes (column mod 8), the slots without
    a photon holding the zero column of the slot's class; from step D_q on
    lane 8 q + f holds zero column f; the quarter warp's own group count is
    ceil(D_q / 4) and each (set, part) range has the largest of the four;
    frames in decreasing photon order, grouped as the host restatement of
    rspi_sets_group groups them (set_order 'grouped') or rank 32 s + p + 4 f
    in lane 8 p + f ('rank'); column of frame d = its slot."""
    size = 37
    d = random_photons(size, n, 40. * size, 15, empty_frames=(2, 9), heavy=5)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, False)
    sx, sy, dia, _ = E.generate_states(E.parse_triple('0 0 1'), E.parse_triple('0 0 1'),
                                       E.parse_triple('2 2 1'))
    es = _estep(_photons(ds, False), size, 3, sx, sy, dia, ds['bg'], form='screen',
                kernel='sets', screen_parts=parts, set_order=set_order)
    torch.cuda.synchronize()
    w = es.wide
    pw, ns = w['part_w'], w['n_sets']
    assert w['n_parts'] == parts and pw % 8 == 0 and parts * pw >= es.p_row - 32
    ent = w['entries'].cpu().numpy().view(np.uint16).reshape(-1, 32, 4).astype(np.int64)
    goff = w['group_off'].cpu().numpy()
    sf = w['set_frames'].cpu().numpy()
    cof = es.col_of_frame.cpu().numpy()
    assert goff.size == parts * ns + 1 and np.all(np.diff(goff) >= 0)
    photons = frame_photons16(es)
    tot = np.array([p.size for p in photons])
    order = np.argsort(-tot, kind='stable')
    k = np.arange(ns * 32)
    if set_order == 'rank':
        src = (k - k % 32) + (k % 32) // 8 + 4 * (k % 8)
        want_sf = np.where(src < n, order[np.minimum(src, n - 1)], -1)
    else:
        from rspi.device import SETS_SWEEPS
        from sets_group_ref import group_frames
        cnt = np.zeros((n, 32), np.int64)
        for fr, ph in enumerate(photons):
            for h in range(parts):
                cnt[fr, 8 * h:8 * h + 8] = np.bincount(ph[ph // pw == h] % pw % 8, minlength=8)
        assert np.array_equal(cnt, w['counts'].cpu().numpy().reshape(n, 32))
        want_sf = group_frames(cnt, order, parts, SETS_SWEEPS)
    assert np.array_equal(sf, want_sf)
    assert np.array_equal(cof[sf[sf >= 0]], k[sf >= 0])
    for s in range(ns):
        for h in range(parts):
            blk = ent[goff[h * ns + s]:goff[h * ns + s + 1]]          # (G, 32, 4)
            steps = blk.transpose(0, 2, 1).reshape(-1, 32)           # (4G, 32)
            assert np.all(steps <= pw + 7)
            qg = w['quarter_groups'].cpu().numpy()[(h * ns + s) * 4:(h * ns + s) * 4 + 4]
            need = 0
            for q in range(4):
                m = np.zeros((8, 8), np.int64)
                for f in range(8):
                    fr = sf[32 * s + 8 * q + f]
                    if fr >= 0:
                        loc = photons[fr][photons[fr] // pw == h] % pw
                        m[f] = np.bincount(loc % 8, minlength=8)
                dq = max(m.sum(1).max(), m.sum(0).max())
                need = max(need, dq)
                assert qg[q] == -(-dq // 4), (s, h, q)
                cls = steps[:dq, 8 * q:8 * q + 8] % 8
                assert all(len(set(row)) == 8 for row in cls), (s, h, q)
                assert np.all(steps[dq:, 8 * q:8 * q + 8] == pw + np.arange(8)), (s, h, q)
            assert blk.shape[0] == -(-need // 4), (s, h)
            for lane in range(32):
                fr = sf[32 * s + lane]
                col = steps[:, lane]
                real = col < pw
                assert np.all(col[~real] == pw + (col[~real] % 8))
                if fr < 0:
                    assert not real.any()
                    continue
                ref = photons[fr][photons[fr] // pw == h] % pw
                assert np.array_equal(np.sort(col[real]), np.sort(ref)), (s, h, lane)


@pytest.mark.parametrize('num_rot,r0,r1', [(5, 0, None), (8, 0, None), (8, 4, 20), (5, 3, 22),
                                           (6, 7, 8)])
def test_sets_slice_layout_bit_identical(num_rot, r0, r1):
    """rspi_rot_log_slices_sets writes the bits of the row-major FP32 slices
    (rspi_rot_log_slices_pairs) in the tile-interleaved part layout, for
    row ranges that start and end inside a state's rotations, with the same
    abs_max."""
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    g = load_golden('case_b')
    ds = golden_dataset(g)
    size = int(g['size'])
    sx, sy, dia, _ = golden_states(g)
    es = _estep(_photons(ds, bool(g['need_scaling'])), size, num_rot, sx, sy, dia, ds['bg'],
                form='screen', kernel='sets', screen_parts=2)
    es.slices(torch.from_numpy(g['model_in_1']).cuda())
    r1 = es.n_rows if r1 is None else r1
    parts, pw = es.wide['n_parts'], es.wide['part_w']
    ref = torch.full((r1 - r0, es.p_row), 7., dtype=torch.float32, device='cuda')
    amax_a = torch.zeros(1, dtype=torch.float32, device='cuda')
    call('rspi_rot_log_slices_pairs', ptr(es.holo_pairs), es.n_states0, es.num_rot,
         ptr(es.rot_cs), es.size, ptr(es.bg), ptr(es.sel_pix), es.n_sel, es.p_row, r0, r1,
         ptr(ref), 0, ptr(amax_a), cur_stream())
    tiles = (r1 - r0 + 3) // 4
    out = torch.full((tiles * parts * pw * 4,), 7., dtype=torch.float32, device='cuda')
    amax_b = torch.zeros(1, dtype=torch.float32, device='cuda')
    call('rspi_rot_log_slices_sets', ptr(es.holo_pairs), None, es.n_states0, es.num_rot,
         ptr(es.rot_cs), es.size, ptr(es.bg), ptr(es.sel_pix), es.n_sel, parts, pw, r0, r1,
         ptr(out), ptr(amax_b), cur_stream())
    torch.cuda.synchronize()
    a = ref.cpu().numpy()
    b = out.cpu().numpy().reshape(tiles, parts, pw, 4)
    for r in range(r1 - r0):
        row = b[r // 4, :, :, r % 4].reshape(-1)           # parts * pw columns
        want = np.zeros(parts * pw, np.float32)
        want[:es.n_sel] = a[r, :es.n_sel]
        assert np.array_equal(row.view(np.uint32), want.view(np.uint32)), r
    assert float(amax_a.item()) == float(amax_b.item()) > 0.


def test_sets_fused_frame_maximum():
    """The screened maximum and first-index argmax folded into the frame-set
    kernel's stores equal those of the FP32 matrix it wrote."""
    g = load_golden('case_b')
    _, es = _golden_estep(g, form='screen', kernel='sets')
    es.run(torch.from_numpy(g['model_in_2']).cuda())
    m = es.frame_prob().cpu().numpy()   # before the rescoring refines candidates
    es.reduce()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(es.rmax32.cpu().numpy(), np.argmax(m, 0))
    np.testing.assert_array_equal(es.max32.cpu().numpy(), m.max(0).astype(np.float64))
    assert not bool(es.frame_max.any())   # reset for the next pass


@pytest.mark.parametrize('delta', [0., 20., 400.])
def test_one_pass_candidates_equal_two_pass(delta):
    """The one-pass candidate selection (counting pass records each thread's
    first two candidates, compaction, a second scan only for frames where a
    thread met more) gives the two-pass lists, in the same order, for
    windows from the argmax alone to hundreds of candidates per frame."""
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    g = load_golden('case_b')
    _, es = _golden_estep(g, form='screen', kernel='sets', delta=delta)
    es.run(torch.from_numpy(g['model_in_1']).cuda())
    es.reduce()                      # sizes the candidate buffers
    n = es.ph.num_data
    outs = []
    for slot in (es.cand_slot, None):
        cand_n = torch.empty(n, dtype=torch.int32, device='cuda')
        off = torch.empty(n + 1, dtype=torch.int64, device='cuda')
        cd = torch.full((es.capacity,), -7, dtype=torch.int32, device='cuda')
        cr = torch.full((es.capacity,), -7, dtype=torch.int32, device='cuda')
        call('rspi_screen_candidates_cols', ptr(es.prob), es.n_rows, es.n_cols,
             ptr(es.frame_of_col), n, ptr(es.max32), ptr(es.rmax32),
             ptr(es.ll['frame_sel_photons']), ptr(es._eps_rows()), ptr(es.lmax), es.delta,
             ptr(es.cnt_part), ptr(cand_n), ptr(es.noncand), ptr(es.thr), ptr(off),
             es.capacity, ptr(cd), ptr(cr), ptr(slot), ptr(es.ph.err.t), cur_stream())
        torch.cuda.synchronize()
        es.ph.err.check('candidates')
        total = int(off[n])
        outs.append((off.cpu().numpy(), cd[:total].cpu().numpy(), cr[:total].cpu().numpy()))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    off, cd, _ = outs[0]
    assert np.array_equal(cd, np.repeat(np.arange(n), np.diff(off)))
    if delta >= 20.:
        # some frames took the second scan (more than 64 candidates: some
        # thread met three or more)
        assert (np.diff(outs[0][0]) > 64).any() or delta == 20.


@pytest.mark.parametrize('name,ds,need_scaling', CASES, ids=[c[0] for c in CASES])
def test_sets_fp32_slice_arithmetic(name, ds, need_scaling):
    """FP32 interpolation and log in the frame-set slices: every value within
    2^-24 (16 + 7|L|) of the FP64 value (the sentinel exactly where FP64 has
    it), the FP32 likelihoods within 1e-5 of the FP64 form's, and after
    FP64 rescoring the same argmax, maximum and log-sum-exp."""
    size = int(round(np.sqrt(ds['num_pix'])))
    num_rot = 6
    sx, sy, dia, _ = E.generate_states(E.parse_triple('-1 1 3'), E.parse_triple('0 1 2'),
                                       E.parse_triple('2 3 2'))
    rng = np.random.default_rng(size + 3)
    model = torch.from_numpy(rng.random(size * size) + 1j * rng.random(size * size)).cuda()
    out = {}
    for math in ('fp64', 'fp32'):
        ph = _photons(ds, need_scaling)
        es = _estep(ph, size, num_rot, sx, sy, dia, ds['bg'], form='screen', kernel='sets',
                    slice_math=math, screen_parts=2 if size > 20 else None)
        es.run(model)
        lsl = es.lsl.clone()
        maxll, rmax, logz = es.reduce()
        torch.cuda.synchronize()
        out[math] = (lsl.cpu().numpy(), es.frame_prob().cpu().numpy().astype(np.float64),
                     maxll.cpu().numpy(), rmax.cpu().numpy(), logz.cpu().numpy())
    a, b = out['fp64'], out['fp32']
    real = a[0] != 0
    assert np.array_equal(a[0] == -1000., b[0] == -1000.)
    assert np.all(np.abs(b[0] - a[0]) <= 2. ** -24 * (16. + 7. * np.abs(a[0])) * (1 + 1e-6))
    assert real.any()
    _, pm = E.generate_masks(size)
    ref = _estep(_photons(ds, need_scaling), size, num_rot, sx, sy, dia, ds['bg'], form='fp64')
    ref.run(model)
    ref.reduce()
    want = ref.frame_prob().cpu().numpy()
    with np.errstate(invalid='ignore'):
        rel = np.abs(b[1] - want) / np.abs(want)
    assert np.nanmax(rel) <= RTOL_F32 or np.isnan(want).all()
    assert np.array_equal(a[3], b[3])
    np.testing.assert_allclose(a[2], b[2], rtol=1e-15)
    np.testing.assert_allclose(a[4], b[4], rtol=1e-9)


@pytest.mark.parametrize('parts', [2, 3])
def test_sets_kernel_beyond_tensor_memory_sets(parts):
    """More than 512 sets (16,384 frames): the running part sums of the
    first 512 sets live in tensor memory, the others in the global scratch;
    every FP32 likelihood within the screening bound eps_d of the FP64
    form's, and the FP64-rescored argmax and maximum equal the FP64 form's,
    for two and three column parts (the middle part reads and rewrites its
    running sums)."""
    size, n = 29, 16384 + 32 * 9 + 5          # 522 sets, the last one partial
    d = random_photons(size, n, 150., 21, empty_frames=(3, n - 1))
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, True)
    sx, sy, dia, _ = E.generate_states(E.parse_triple('-1 1 2'), E.parse_triple('0 0 1'),
                                       E.parse_triple('2 2 1'))
    num_rot = 4
    rng = np.random.default_rng(7)
    model = torch.from_numpy(rng.random(size * size) + 1j * rng.random(size * size)).cuda()
    ref = _estep(_photons(ds, True), size, num_rot, sx, sy, dia, ds['bg'], form='fp64')
    ref.run(model)
    maxll64, rmax64, _ = ref.reduce()
    want = ref.frame_prob().cpu().numpy()
    ph = _photons(ds, True)
    es = _estep(ph, size, num_rot, sx, sy, dia, ds['bg'], form='screen', kernel='sets',
                screen_parts=parts)
    assert es.wide['n_sets'] > 512 and es.wide['n_parts'] == parts
    es.run(model)
    maxll, rmax, _ = es.reduce()
    torch.cuda.synchronize()
    ph.err.check('sets kernel beyond the tensor-memory sets')
    got = es.frame_prob().cpu().numpy().astype(np.float64)
    rows = np.diff(es._eps_rows().cpu().numpy()).astype(np.float64)
    phot = es.ll['frame_sel_photons'].cpu().numpy().astype(np.float64)
    lmax = float(es.lmax.cpu().numpy().reshape(-1)[0])
    eps = 2. ** -24 * ((rows + 8.) * phot * lmax + np.abs(want) + 1.)
    err = np.abs(got - want)
    worst = np.unravel_index(np.argmax(err / eps), err.shape)
    assert np.all(err <= eps), (worst, err[worst], eps[worst])
    assert np.array_equal(rmax.cpu().numpy(), rmax64.cpu().numpy())
    np.testing.assert_allclose(maxll.cpu().numpy(), maxll64.cpu().numpy(), rtol=1e-14)


@pytest.mark.parametrize('delta', [0., 20.])
def test_candidates_many_rows(delta):
    """18 states x 180 rotations (3,240 likelihood rows), frames in set
    order: the one-pass selection gives the second scan's lists, and the
    rescored argmax and maximum equal the FP64 form's; the log-sum-exp too,
    to 1e-12 with a 20-nat window, and within the FP32 error of the
    non-candidates' terms (1e-7) with the argmax alone."""
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    size, n, num_rot = 37, 300, 180
    d = random_photons(size, n, 30. * size, 41, empty_frames=(3,), heavy=7)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, True)
    sx, sy, dia, _ = E.generate_states(E.parse_triple('-1 1 3'), E.parse_triple('-1 1 3'),
                                       E.parse_triple('2 3 2'))
    rng = np.random.default_rng(5)
    model = torch.from_numpy(rng.random(size * size) + 1j * rng.random(size * size)).cuda()
    es = _estep(_photons(ds, True), size, num_rot, sx, sy, dia, ds['bg'], form='screen',
                kernel='sets', delta=delta)
    ref = _estep(_photons(ds, True), size, num_rot, sx, sy, dia, ds['bg'], form='fp64')
    assert es.n_rows == 3240
    es.run(model)
    ref.run(model)
    maxll, rmax, logz = es.reduce()
    ref.reduce()
    torch.cuda.synchronize()
    assert np.array_equal(rmax.cpu().numpy(), ref.rmax.cpu().numpy())
    np.testing.assert_allclose(maxll.cpu().numpy(), ref.maxll.cpu().numpy(), rtol=1e-15)
    np.testing.assert_allclose(logz.cpu().numpy(), ref.logz.cpu().numpy(),
                               rtol=1e-12 if delta >= 20. else 1e-7)
    outs = []
    for slot in (es.cand_slot, None):
        cand_n = torch.empty(n, dtype=torch.int32, device='cuda')
        off = torch.empty(n + 1, dtype=torch.int64, device='cuda')
        cd = torch.full((es.capacity,), -7, dtype=torch.int32, device='cuda')
        cr = torch.full((es.capacity,), -7, dtype=torch.int32, device='cuda')
        call('rspi_screen_candidates_cols', ptr(es.prob), es.n_rows, es.n_cols,
             ptr(es.frame_of_col), n, ptr(es.max32), ptr(es.rmax32),
             ptr(es.ll['frame_sel_photons']), ptr(es._eps_rows()), ptr(es.lmax), es.delta,
             ptr(es.cnt_part), ptr(cand_n), ptr(es.noncand), ptr(es.thr), ptr(off),
             es.capacity, ptr(cd), ptr(cr), ptr(slot), ptr(es.ph.err.t), cur_stream())
        torch.cuda.synchronize()
        es.ph.err.check('candidates')
        total = int(off[n])
        outs.append((off.cpu().numpy(), cd[:total].cpu().numpy(), cr[:total].cpu().numpy()))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    assert int(outs[0][0][-1]) >= n   # at least each frame's argmax
