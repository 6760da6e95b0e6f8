"""NumPy restatement of the frame grouping of the frame-set kernel
(rspi_sets_group, csrc/ll_sets.cu): the same greedy quarters, pair sweeps
and quarter order, with the same tie rules, so that the GPU result can be
compared element for element.  Test infrastructure only."""
import numpy as np

WINDOW = 256   # frames per window (GROUP_W)


def quarter_cost(c):
    """c: (..., 8 frames, parts, 8 classes) -> sum over parts of
    max(largest frame, largest class total)."""
    lane = c.sum(-1).max(-2)
    cls = c.sum(-3).max(-1)
    return np.maximum(lane, cls).sum(-1)


def group_window(cnt, sweeps):
    """Quarters (local indices, -1 empty) of one window, in set order."""
    m = cnt.shape[0]
    nq = -(-m // 8)
    length = cnt.sum(-1)
    used = np.zeros(m, bool)
    q8 = np.full((nq, 8), -1, np.int64)
    for q in range(nq):
        free = np.flatnonzero(~used)
        if free.size == 0:
            break
        f = int(free[0])
        q8[q, 0] = f
        used[f] = True
        s, lmax = cnt[f].copy(), length[f].copy()
        for k in range(1, 8):
            free = np.flatnonzero(~used)
            if free.size == 0:
                break
            cost = np.maximum(np.maximum(lmax[None], length[free]),
                              (s[None] + cnt[free]).max(-1)).sum(-1)
            f = int(free[np.argmin(cost)])          # first minimum: the lower rank
            q8[q, k] = f
            used[f] = True
            s += cnt[f]
            lmax = np.maximum(lmax, length[f])
    cz = np.concatenate([cnt, np.zeros((1,) + cnt.shape[1:], cnt.dtype)])   # -1: no photons
    qc = quarter_cost(cz[q8])
    ii, jj = np.divmod(np.arange(64), 8)
    rows = np.arange(64)
    for _ in range(sweeps):
        changed = False
        for a in range(nq):
            for b in range(a + 1, nq):
                fa, fb = q8[a][ii], q8[b][jj]
                qa = np.repeat(q8[a][None], 64, 0)
                qb = np.repeat(q8[b][None], 64, 0)
                qa[rows, ii] = fb
                qb[rows, jj] = fa
                ca, cb = quarter_cost(cz[qa]), quarter_cost(cz[qb])
                delta = ca + cb - qc[a] - qc[b]
                delta[(fa < 0) & (fb < 0)] = 0
                t = int(np.argmin(delta))               # ties: the lower exchange index
                if delta[t] < 0:
                    q8[a], q8[b] = qa[t], qb[t]
                    qc[a], qc[b] = ca[t], cb[t]
                    changed = True
        if not changed:
            break
    return q8[np.argsort(-qc, kind='stable')]


def group_frames(counts, order, n_parts, sweeps):
    """set_frames (ceil(n / 32) * 32, -1 empty) for counts (n x 32 ints:
    part h, class c at h * 8 + c) and the frames by decreasing photon
    count."""
    counts = np.asarray(counts).reshape(-1, 32)[:, :n_parts * 8].reshape(-1, n_parts, 8)
    order = np.asarray(order, dtype=np.int64)
    out = []
    for w0 in range(0, order.size, WINDOW):
        idx = order[w0:w0 + WINDOW]
        q8 = group_window(counts[idx].astype(np.int64), sweeps)
        frames = np.where(q8 >= 0, idx[np.maximum(q8, 0)], -1)
        ns = -(-q8.shape[0] // 4)
        pad = np.full((ns * 4 - q8.shape[0], 8), -1, np.int64)
        out.append(np.concatenate([frames, pad]).reshape(-1))
    return np.concatenate(out)
