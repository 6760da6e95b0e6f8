"""The frame-grouping restatement on the host: a set layout holding every
frame once, deterministic, and no dearer than the rank order."""
import numpy as np

from sets_group_ref import group_frames, quarter_cost


def test_restatement_is_a_set_layout_and_cheaper():
    rng = np.random.default_rng(1)
    n, parts = 300, 2
    c = np.zeros((n, 32), np.int64)
    c[:, :16] = rng.poisson(rng.lognormal(np.log(40.), 0.5, n)[:, None] / 8., (n, 16))
    order = np.argsort(-c.sum(1), kind='stable')
    sf = group_frames(c, order, parts, 2)
    assert sf.size == -(-n // 32) * 32
    assert np.array_equal(np.sort(sf[sf >= 0]), np.arange(n))
    assert np.array_equal(sf, group_frames(c, order, parts, 2))
    cz = np.concatenate([c[:, :16].reshape(n, parts, 8), np.zeros((1, parts, 8), np.int64)])
    k = np.arange(sf.size)
    lane = k % 32
    src = (k - lane) + lane // 8 + 4 * (lane % 8)
    rank = np.where(src < n, order[np.minimum(src, n - 1)], -1)
    assert quarter_cost(cz[sf.reshape(-1, 8)]).sum() < quarter_cost(cz[rank.reshape(-1, 8)]).sum()
