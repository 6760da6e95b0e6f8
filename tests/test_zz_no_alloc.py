"""The no-allocation candidate entry point against the regular one.

rspi_screen_candidates_noalloc serves callers that cannot allocate device
memory (they cannot hand the library a scratch buffer): it keeps its scratch
in a fixed array inside librspi.so.  This test calls it through the C ABI
twice in a row on the same screened likelihoods and checks every output
against rspi_screen_candidates given caller-owned scratch.  The file sorts
last so that a run stopping at the first failure has run every other test.
"""
import numpy as np
import pytest
import torch

from helpers import golden_dataset, golden_states, load_golden
from oracle import emc_oracle as E

pytestmark = pytest.mark.gpu


def _screened():
    from rspi.device import DevicePhotons, EStep, call, cur_stream, ptr
    g = load_golden('case_b')
    ds = golden_dataset(g)
    size, num_rot = int(g['size']), int(g['num_rot'])
    sx, sy, dia, _ = golden_states(g)
    ph = DevicePhotons(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                       ds['count_multi'], ds['num_pix'], bool(g['need_scaling']))
    _, pm = E.generate_masks(size)
    es = EStep(ph, size, num_rot, sx, sy, dia, pm, ds['bg'], form='screen', kernel='stream')
    es.run(torch.from_numpy(g['model_in_1']).cuda())
    call('rspi_frame_reduce', ptr(es.prob), 0, es.n_rows, ph.num_data, ptr(es.max32),
         ptr(es.rmax32), None, cur_stream())
    return es


def _outputs(es):
    n, cap = es.ph.num_data, es.capacity
    dev = es.device
    return dict(cand_n=torch.full((n,), -7, dtype=torch.int32, device=dev),
                noncand=torch.full((n,), -7., dtype=torch.float64, device=dev),
                thr=torch.full((n,), -7., dtype=torch.float64, device=dev),
                cand_off=torch.full((n + 1,), -7, dtype=torch.int64, device=dev),
                cand_d=torch.full((cap,), -7, dtype=torch.int32, device=dev),
                cand_r=torch.full((cap,), -7, dtype=torch.int32, device=dev),
                err=torch.zeros(1, dtype=torch.int32, device=dev))


def _common_args(es):
    from rspi.device import ptr
    return (ptr(es.prob), es.n_rows, es.ph.num_data, ptr(es.max32), ptr(es.rmax32),
            ptr(es.ll['frame_sel_photons']), ptr(es.ll16['row_off']), ptr(es.lmax), es.delta)


def test_noalloc_candidates_match_allocating_entry_point():
    from rspi.device import call, cur_stream, ptr
    es = _screened()
    n = es.ph.num_data
    ref = _outputs(es)
    scratch = torch.empty(n * 32, dtype=torch.int32, device=es.device)
    call('rspi_screen_candidates', *_common_args(es), ptr(scratch), ptr(ref['cand_n']),
         ptr(ref['noncand']), ptr(ref['thr']), ptr(ref['cand_off']), es.capacity,
         ptr(ref['cand_d']), ptr(ref['cand_r']), ptr(ref['err']), cur_stream())
    torch.cuda.synchronize()
    total = int(ref['cand_off'][n])
    assert 0 < total <= es.capacity and int(ref['err']) == 0
    for _ in range(2):   # two calls in a row share the library's scratch
        out = _outputs(es)
        call('rspi_screen_candidates_noalloc', *_common_args(es), ptr(out['cand_n']),
             ptr(out['noncand']), ptr(out['thr']), ptr(out['cand_off']), es.capacity,
             ptr(out['cand_d']), ptr(out['cand_r']), ptr(out['err']), cur_stream())
        torch.cuda.synchronize()
        assert int(out['err']) == 0
        for key in ('cand_n', 'cand_off'):
            assert torch.equal(out[key], ref[key]), key
        for key in ('noncand', 'thr'):
            np.testing.assert_allclose(out[key].cpu().numpy(), ref[key].cpu().numpy(),
                                       rtol=1e-12, atol=0)
        for key in ('cand_d', 'cand_r'):
            assert torch.equal(out[key][:total], ref[key][:total]), key


def test_noalloc_rejects_more_frames_than_its_scratch():
    from rspi.lib import load
    lib = load()
    null = None
    code = lib.rspi_screen_candidates_noalloc(null, 1, 65537, null, null, null, null, null, 20.,
                                              null, null, null, null, 0, null, null, null, null)
    assert code == -6
    assert 'scratch' in lib.rspi_status_string(code).decode()


def test_noalloc_at_its_frame_limit():
    """65,536 frames, the most the fixed scratch holds: the last slots of the
    library's array are written and read back, and the outputs equal the
    allocating entry point's on a synthetic likelihood matrix."""
    from rspi.device import call, cur_stream, ptr
    n, rows = 65536, 9
    g = torch.Generator(device='cuda')
    g.manual_seed(5)
    ll = (torch.randn((rows, n), generator=g, device='cuda') * 3. - 100.).float()
    max32 = torch.empty(n, dtype=torch.float64, device='cuda')
    rmax32 = torch.empty(n, dtype=torch.int32, device='cuda')
    call('rspi_frame_reduce', ptr(ll), 0, rows, n, ptr(max32), ptr(rmax32), None, cur_stream())
    phot = torch.randint(0, 300, (n,), generator=g, device='cuda', dtype=torch.int64)
    row_off = torch.arange(n + 1, device='cuda', dtype=torch.int64) * 4
    lmax = torch.ones(1, dtype=torch.float32, device='cuda')
    cap = rows * n

    def outputs():
        return dict(cand_n=torch.full((n,), -7, dtype=torch.int32, device='cuda'),
                    noncand=torch.full((n,), -7., dtype=torch.float64, device='cuda'),
                    thr=torch.full((n,), -7., dtype=torch.float64, device='cuda'),
                    cand_off=torch.full((n + 1,), -7, dtype=torch.int64, device='cuda'),
                    cand_d=torch.full((cap,), -7, dtype=torch.int32, device='cuda'),
                    cand_r=torch.full((cap,), -7, dtype=torch.int32, device='cuda'),
                    err=torch.zeros(1, dtype=torch.int32, device='cuda'))
    common = (ptr(ll), rows, n, ptr(max32), ptr(rmax32), ptr(phot), ptr(row_off), ptr(lmax),
              2.0)
    ref = outputs()
    scratch = torch.empty(n * 32, dtype=torch.int32, device='cuda')
    call('rspi_screen_candidates', *common, ptr(scratch), ptr(ref['cand_n']),
         ptr(ref['noncand']), ptr(ref['thr']), ptr(ref['cand_off']), cap, ptr(ref['cand_d']),
         ptr(ref['cand_r']), ptr(ref['err']), cur_stream())
    torch.cuda.synchronize()
    total = int(ref['cand_off'][n])
    assert total > n and int(ref['err']) == 0
    for _ in range(2):
        out = outputs()
        call('rspi_screen_candidates_noalloc', *common, ptr(out['cand_n']), ptr(out['noncand']),
             ptr(out['thr']), ptr(out['cand_off']), cap, ptr(out['cand_d']), ptr(out['cand_r']),
             ptr(out['err']), cur_stream())
        torch.cuda.synchronize()
        assert int(out['err']) == 0
        for key in ('cand_n', 'cand_off'):
            assert torch.equal(out[key], ref[key]), key
        for key in ('cand_d', 'cand_r'):
            assert torch.equal(out[key][:total], ref[key][:total]), key
        for key in ('noncand', 'thr'):
            np.testing.assert_allclose(out[key].cpu().numpy(), ref[key].cpu().numpy(),
                                       rtol=1e-12, atol=0)
