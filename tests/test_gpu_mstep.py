"""MaxLP M-step parity on the GPU (rows a11-a14) and the end-to-end EMC
iteration against the reference goldens."""
import os

import numpy as np
import pytest
import torch

from helpers import GOLDEN_CASES, golden_dataset, load_golden, random_photons, write_case
from oracle import emc_oracle as E
from oracle import maxlp_oracle as M

pytestmark = pytest.mark.gpu

RTOL_MODEL = 1e-9   # FP64 pattern search: same path, rounding-level differences


def _photons(ds, need_scaling=False):
    from rspi.device import DevicePhotons
    return DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                         ds['count_multi'], ds['num_pix'], need_scaling)


@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_histogram_bit_exact(name):
    """hist[t][s] == sum over frames in state s of the oracle's k_d(t)."""
    from rspi import geometry
    from rspi.device import MStep
    g = load_golden(name)
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    rmax = g['rmax_1']
    n_ref = int(g['prob_1'].shape[0] // num_rot)
    ph = _photons(ds)
    ms = MStep(ph, size)
    ms.frame_params_from_rmax(torch.from_numpy(rmax).cuda(), num_rot, n_ref)
    ang = (rmax % num_rot) * np.pi / num_rot
    rot = torch.from_numpy(geometry.phaser_rotation_table(np.arange(num_rot) * np.pi / num_rot)).cuda()
    ms.hist = torch.zeros(ms.n_hist_rows * n_ref, dtype=torch.int32, device='cuda')
    from rspi.device import ptr, cur_stream
    from rspi.lib import check
    check(ms.lib.rspi_maxlp_histogram(
        ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum), ptr(ph.multi_accum), ptr(ph.place_ones),
        ptr(ph.place_multi), ptr(ph.count_multi), ph.num_data, ptr(ms.fstate), ptr(ms.frot),
        ptr(rot), size, ptr(ms.mask_idx), ms.n_hist_rows, n_ref, ptr(ms.hist), ptr(ph.err.t),
        cur_stream()), 'hist')
    hist = ms.hist.cpu().numpy().reshape(ms.n_hist_rows, n_ref)
    assert np.array_equal(ms.nstate.cpu().numpy(), np.bincount(rmax // num_rot, minlength=n_ref))
    kmat = E.sparse_frames(ds)
    qx, qy, _, mask, rmask = M.get_qvals(size)
    rows = np.flatnonzero(mask | rmask)
    fstate = rmax // num_rot
    for m, t in enumerate(rows):
        k = M.photons_pixel(kmat, ang, int(t), size, qx, qy)
        want = np.bincount(fstate, weights=k, minlength=n_ref).astype(np.int64)
        assert np.array_equal(hist[m], want), t


@pytest.mark.parametrize('name', GOLDEN_CASES)
@pytest.mark.parametrize('it', [1, 2])
def test_run_phaser_matches_reference(name, it, tmp_path):
    """MaxLPhaser._run_phaser (generic per-frame parameters) vs the goldens."""
    from maxLP import MaxLPhaser
    g = load_golden(name)
    cfg = write_case(str(tmp_path), g)
    ph = MaxLPhaser(os.path.join(str(tmp_path), 'photons.npz'), size=int(g['size']))
    out = ph._run_phaser(g['model_in_%d' % it], *g['unravel_%d' % it])
    np.testing.assert_allclose(out, g['model_out_%d' % it], rtol=RTOL_MODEL, atol=1e-12)
    del cfg


@pytest.mark.parametrize('form', ['fp64', 'screen'])
@pytest.mark.parametrize('name', GOLDEN_CASES)
def test_emc_two_iterations_match_reference(name, form, tmp_path):
    from emc import EMC
    g = load_golden(name)
    cfg = write_case(str(tmp_path), g, extra='form = %s\n' % form)
    rec = EMC(cfg)
    rec.model = g['model_in_1'].copy()
    for it in (1, 2):
        np.testing.assert_allclose(rec.model, g['model_in_%d' % it], rtol=RTOL_MODEL, atol=1e-12)
        rec.run_iteration(it)
        np.testing.assert_allclose(rec.prob.cpu().numpy(), g['prob_%d' % it],
                                   rtol=1e-10 if form == 'fp64' else 1e-5)
        assert np.array_equal(rec.rmax, g['rmax_%d' % it])
        np.testing.assert_allclose(np.stack(rec._unravel_rmax(rec.rmax)), g['unravel_%d' % it],
                                   rtol=0, atol=0)
        np.testing.assert_allclose(rec.model, g['model_out_%d' % it], rtol=RTOL_MODEL, atol=1e-12)
        from rspi import h5lite
        out = h5lite.read_datasets(os.path.join(str(tmp_path), 'out', 'output_%03d.h5' % it))
        assert out['model'].shape == (int(g['size']),) * 2
        if it == 2:   # the last file holds the final model
            np.testing.assert_array_equal(out['model'], rec.model.reshape(out['model'].shape))
        np.testing.assert_array_equal(out['angles'], g['unravel_%d' % it][3])
        np.testing.assert_array_equal(out['shifts'], g['unravel_%d' % it][:2].T)


@pytest.mark.parametrize('size', [5, 17, 23])
def test_phaser_random_vs_oracle(size, tmp_path):
    """Odd sizes including a ring-only detector (size 5: empty main mask)."""
    from maxLP import MaxLPhaser
    from rspi.photonfile import write_photons
    n = 24
    d = random_photons(size, n, 20. * size, 10 + size, empty_frames=(2,))
    path = os.path.join(str(tmp_path), 'p.npz')
    write_photons(path, d)
    rng = np.random.default_rng(size)
    sx = rng.choice([-1., 0., 1.], n)
    sy = rng.choice([0., 1.], n)
    dia = rng.choice([2., 3.], n)
    ang = rng.integers(0, 6, n) * np.pi / 6
    model = rng.random(size * size) + 1j * rng.random(size * size)
    ph = MaxLPhaser(path, size=size)
    got = ph._run_phaser(model, sx, sy, dia, ang)
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size)
    with np.errstate(invalid='ignore', divide='ignore'):
        want = M.run_phaser(model, E.sparse_frames(ds), sx, sy, dia, ang, size)
    np.testing.assert_allclose(got, want, rtol=RTOL_MODEL, atol=1e-12)


@pytest.mark.parametrize('form', ['fp64', 'screen'])
def test_emc_graph_replay_matches_eager(form, tmp_path):
    """Three iterations replayed from the captured CUDA graph give exactly the
    eager iterations' rmax and model."""
    from emc import EMC
    g = load_golden('case_a')
    out = {}
    for graph in (False, True):
        d = os.path.join(str(tmp_path), str(graph))
        cfg = write_case(d, g, extra='form = %s\ncuda_graph = %s\n' % (form, graph))
        rec = EMC(cfg)
        rec.model = g['model_in_1'].copy()
        hist = []
        for it in range(3):
            rec.run_iteration(None)
            hist.append((rec.rmax.copy(), rec.model.copy()))
        assert (rec._graph is not None) == graph
        out[graph] = hist
    for (ra, ma), (rb, mb) in zip(out[False], out[True]):
        assert np.array_equal(ra, rb)
        assert np.array_equal(ma, mb)


def test_recon_cli_writes_log_and_outputs(tmp_path):
    """recon.py keeps the reference CLI and EMC.log format (recon.py:16-65)."""
    import recon
    g = load_golden('case_a')
    cfg = write_case(str(tmp_path), g)
    rec = recon.main(['2', '-c', cfg])
    log = open(os.path.join(str(tmp_path), 'out', 'EMC.log')).read().splitlines()
    assert log[0] == 'Iter  time(s)  change' and len(log) == 3
    assert log[1].split()[0] == '1' and log[2].split()[0] == '2'
    from rspi import h5lite
    n = len(g['ones'])
    grid = np.arange(int(g['num_rot'])) * np.pi / int(g['num_rot'])
    for it in (1, 2):
        out = h5lite.read_datasets(os.path.join(str(tmp_path), 'out', 'output_%03d.h5' % it))
        assert out['model'].shape == (int(g['size']),) * 2
        assert out['angles'].shape == out['diameters'].shape == (n,)
        assert out['shifts'].shape == (n, 2)
        assert np.all(np.isin(out['angles'], grid))
    # the last file holds the final model and the last iteration's states
    sxv, syv, diav, angv = rec._unravel_rmax(rec.rmax)
    np.testing.assert_array_equal(out['model'], rec.model.reshape(out['model'].shape))
    np.testing.assert_array_equal(out['angles'], angv)
    np.testing.assert_array_equal(out['diameters'], diav)
    np.testing.assert_array_equal(out['shifts'], np.array([sxv, syv]).T)
    assert os.path.exists(os.path.join(str(tmp_path), 'out', 'model_000.npy'))
    assert rec.rmax.shape == (len(g['ones']),)


@pytest.mark.parametrize('kind', ['grid', 'lbfgs', 'grid+lbfgs'])
def test_emc_adjoint_driven_mstep(tmp_path, kind):
    """[emc] mstep = grid / lbfgs / grid+lbfgs: the E-step (replayed from its
    CUDA graph after the first iteration) gives the reference's argmax, the
    M-step keeps the ring pass of the pattern search and then lowers the
    pixel NLL of the main pixels below that of its start (the model after the
    ring pass); the grid followed by L-BFGS goes below the pattern search's
    (the 64 x 32 polar grid alone, or 20 L-BFGS steps alone from the start,
    need not); iterations run through EMC.run_iteration."""
    from emc import EMC
    from rspi.adjoint import NLLProblem
    g = load_golden('case_b')
    cfg = write_case(str(tmp_path), g=g, extra='mstep = %s\nlbfgs_steps = 20\n' % kind)
    rec = EMC(cfg)
    assert rec.mstep_kind == kind
    rec.model = g['model_in_1'].copy()
    rec.run_iteration(1)
    assert np.array_equal(rec.rmax, g['rmax_1'])
    ms = rec.phaser.mstep
    rho = float(ms.rescale[0])
    # the pattern search's model from the same start, for comparison
    ref = EMC(write_case(str(tmp_path / 'p'), g=g))
    ref.model = g['model_in_1'].copy()
    ref.run_iteration(1)
    num_rot = int(g['num_rot'])
    vals = rec.state_vals[ms.fstate.long()]
    ang = (ms.frot.double() * np.pi / num_rot).cpu().numpy()
    prob = NLLProblem(rec.dset.photons, rec.size, ang, precision='fp64')
    scale = rec.dset.photons.scales * rho

    def nll(m):
        fre, fim = prob.model_pixels(m)
        return float(prob.evaluate(fre, fim, vals[:, 2], vals[:, 0], vals[:, 1], scale))
    # the start of the main-pixel search: model_in_1 after the ring pass
    start = torch.from_numpy(g['model_in_1'].copy()).cuda()
    ms.run(start, rec.state_vals, rec.phaser_rot, main=False)
    assert nll(rec.model) < nll(start.cpu().numpy())
    if kind == 'grid+lbfgs':
        assert nll(rec.model) < nll(ref.model)
    # a second iteration replays the E-step graph and runs the M-step eagerly
    rec.run_iteration(2)
    assert rec._graph is not None
    assert np.all(np.isfinite(rec.model))


@pytest.mark.parametrize('size,n,num_rot', [(20, 200, 12), (37, 300, 180), (24, 150, 7)])
def test_pixel_map_histogram_equals_search(size, n, num_rot):
    """The histogram from the per-rotation pixel map (rspi_maxlp_pixel_map +
    rspi_maxlp_histogram_map) equals the per-photon search's
    (rspi_maxlp_histogram) bit for bit, even detectors (the column-`size`
    alias) included, and the oracle's photons per pixel."""
    from rspi import geometry
    from rspi.device import MStep, cur_stream, ptr
    from rspi.lib import check
    from helpers import random_photons
    d = random_photons(size, n, 40. * size, size + n, empty_frames=(1,))
    ds = E.parse_photons(d['ones'], d['multi'], d['place_ones'], d['place_multi'],
                         d['count_multi'], size * size, False)
    rng = np.random.default_rng(size)
    n_ref = 5
    rmax = rng.integers(0, n_ref * num_rot, n).astype('i4')
    ph = _photons(ds)
    ms = MStep(ph, size)
    ms.frame_params_from_rmax(torch.from_numpy(rmax).cuda(), num_rot, n_ref)
    rot = torch.from_numpy(geometry.phaser_rotation_table(np.arange(num_rot) * np.pi / num_rot)).cuda()
    got = ms.histogram(n_ref, rot).clone()
    want = torch.zeros_like(got)
    check(ms.lib.rspi_maxlp_histogram(
        ptr(ph.ones), ptr(ph.multi), ptr(ph.ones_accum), ptr(ph.multi_accum), ptr(ph.place_ones),
        ptr(ph.place_multi), ptr(ph.count_multi), ph.num_data, ptr(ms.fstate), ptr(ms.frot),
        ptr(rot), size, ptr(ms.mask_idx), ms.n_hist_rows, n_ref, ptr(want), ptr(ph.err.t),
        cur_stream()), 'hist')
    torch.cuda.synchronize()
    ph.err.check('histogram')
    assert ms._pixel_map is not None   # the map path ran
    assert torch.equal(got, want)
    hist = got.cpu().numpy().reshape(ms.n_hist_rows, n_ref)
    kmat = E.sparse_frames(ds)
    qx, qy, _, mask, rmask = M.get_qvals(size)
    ang = (rmax % num_rot) * np.pi / num_rot
    fstate = rmax // num_rot
    rows = np.flatnonzero(mask | rmask)
    for m in range(0, rows.size, 7):
        k = M.photons_pixel(kmat, ang, int(rows[m]), size, qx, qy)
        want_m = np.bincount(fstate, weights=k, minlength=n_ref).astype(np.int64)
        assert np.array_equal(hist[m], want_m), rows[m]
