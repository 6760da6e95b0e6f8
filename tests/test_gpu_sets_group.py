"""Frame grouping of the frame-set kernel (rspi_sets_group) against its
NumPy restatement (tests/sets_group_ref.py), element for element; its
output is a set layout holding every frame once; and it lowers the
quarter warps' step counts against the rank order."""
import numpy as np
import pytest
import torch

from sets_group_ref import group_frames, quarter_cost

pytestmark = pytest.mark.gpu


def _counts(n, n_parts, seed, mean=30.):
    rng = np.random.default_rng(seed)
    lam = rng.lognormal(np.log(mean), 0.5, n)
    c = np.zeros((n, 32), np.int32)
    c[:, :n_parts * 8] = rng.poisson(lam[:, None] / 8., (n, n_parts * 8))
    c[rng.integers(0, n, max(1, n // 50))] = 0                 # frames without photons
    c[0, :n_parts * 8] += 40                                   # one heavy frame
    return c


def _gpu_group(c, order, n_parts, sweeps):
    from rspi.device import cur_stream, ptr
    from rspi.lib import call
    n = c.shape[0]
    ct = torch.from_numpy(c).cuda()
    ot = torch.from_numpy(order.astype(np.int32)).cuda()
    out = torch.full((-(-n // 32) * 32,), -7, dtype=torch.int32, device='cuda')
    err = torch.zeros(1, dtype=torch.int32, device='cuda')
    call('rspi_sets_group', ptr(ct), ptr(ot), n, n_parts, sweeps, ptr(out), ptr(err), cur_stream())
    torch.cuda.synchronize()
    return out.cpu().numpy(), int(err.item())


@pytest.mark.parametrize('n,n_parts,sweeps', [(1, 1, 4), (37, 2, 4), (256, 1, 0), (700, 2, 4),
                                              (613, 3, 2), (300, 4, 1)])
def test_grouping_matches_restatement(n, n_parts, sweeps):
    c = _counts(n, n_parts, 7 + n)
    order = np.argsort(-c.sum(1), kind='stable')
    got, err = _gpu_group(c, order, n_parts, sweeps)
    assert err == 0
    want = group_frames(c, order, n_parts, sweeps)
    assert np.array_equal(got, want)
    assert np.array_equal(np.sort(got[got >= 0]), np.arange(n))
    assert np.all(got[got < 0] == -1)


def test_grouping_lowers_quarter_steps():
    n, parts = 2048, 2
    c = _counts(n, parts, 3, mean=120.)
    order = np.argsort(-c.sum(1), kind='stable')
    got, _ = _gpu_group(c, order, parts, 4)
    k = np.arange(got.size)
    lane = k % 32
    src = (k - lane) + lane // 8 + 4 * (lane % 8)
    rank = np.where(src < n, order[np.minimum(src, n - 1)], -1)
    cz = np.concatenate([c[:, :parts * 8].reshape(n, parts, 8), np.zeros((1, parts, 8), np.int32)])
    cost = {name: quarter_cost(cz[sf.reshape(-1, 8)]).sum() for name, sf in
            (('grouped', got), ('rank', rank))}
    print(cost)
    assert cost['grouped'] < 0.95 * cost['rank']


def test_grouping_flags_frames_outside_the_dataset():
    c = _counts(64, 1, 5)
    order = np.argsort(-c.sum(1), kind='stable')
    order[10] = 64
    got, err = _gpu_group(c, order, 1, 1)
    assert err == -2   # RSPI_ERR_INDEX (include/rspi.h)
    assert 64 not in got and (got == -1).sum() == 1


def test_emc_set_order_option_gives_the_same_iteration(tmp_path):
    """[emc] set_order = grouped / rank: the screened likelihood columns are
    grouped differently, the FP64-rescored argmax and the model after the
    M-step are the same bits."""
    import os
    from emc import EMC
    from helpers import load_golden, write_case
    g = load_golden('case_b')
    out = {}
    for order in ('grouped', 'rank'):
        cfg = write_case(os.path.join(str(tmp_path), order), g,
                         extra='form = screen\nkernel = sets\nset_order = %s\n' % order)
        rec = EMC(cfg)
        assert rec.estep.set_order == order
        rec.model = g['model_in_1'].copy()
        rec.run_iteration(None)
        out[order] = (rec.model.copy(), rec.rmax.copy())
    a, b = out['grouped'], out['rank']
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(np.ascontiguousarray(a[0]).view(np.uint8),
                          np.ascontiguousarray(b[0]).view(np.uint8))
