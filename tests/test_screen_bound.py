"""The FP32 summation order of the four-row frame-quad screening kernel
(k_screen_ll7 in csrc/ll_screen2.cu), emulated on the host in float32, stays
within the error the candidate threshold allows for it.

Per column part h and row, lane j of a frame (local column = j mod 8) adds
its photons group by group: slots 0 + 1 into one accumulator and slots 2 + 3
into the other (a frame's groups after its own last photon add the zero pad
column), then a0 + a1, then three exchange steps over the eight lanes (xor 4,
xor 2, xor 1).  The parts' FP32 sums are combined in FP64; with more than two
parts the running sum between parts is stored as float32.  Each photon's
value therefore passes through at most G + 5 + max(0, P - 2) FP32 roundings
(G = the quad's group count in the part), within the rows + 8 of the
threshold's eps_d = 2^-24 ((rows + 8) photons max|L| + ...) with rows >= G.
The test checks the emulated error against that chain on random and
adversarial values."""
import math

import numpy as np

U32 = 2.0 ** -24
F = np.float32


def _lane_sum(vals, n_groups):
    """One lane over n_groups groups of four slots (missing slots are the
    zero column): a0 += v0 + v1, a1 += v2 + v3, then a0 + a1 -- float32."""
    v = np.zeros(4 * n_groups, dtype=F)
    v[:len(vals)] = vals
    a0 = F(0.)
    a1 = F(0.)
    for g in range(n_groups):
        a0 = F(a0 + F(v[4 * g] + v[4 * g + 1]))
        a1 = F(a1 + F(v[4 * g + 2] + v[4 * g + 3]))
    return F(a0 + a1)


def _tree8(x):
    """Lanes 2t, 2t+1 after the xor 4 / xor 2 / xor 1 steps: row sums in the
    kernel's order for a lane j = 4b + 2e: ((x_j + x_j^4) + (x_j^2 + x_j^6))
    + the same for j ^ 1."""
    def half(j):
        return F(F(x[j] + x[j ^ 4]) + F(x[j ^ 2] + x[j ^ 6]))
    j = 0
    return F(half(j) + half(j ^ 1))


def _kernel_sum(values, classes, parts_of, n_parts, groups):
    """Emulated k_screen_ll7 sum of one frame in one row; groups[h] is its
    quad's group count in part h (>= the frame's own)."""
    run = 0.
    for h in range(n_parts):
        lanes = []
        for j in range(8):
            sel = values[(parts_of == h) & (classes == j)]
            lanes.append(_lane_sum(sel, groups[h]))
        s = _tree8(lanes)
        if h == n_parts - 1:
            run = run + float(s)                       # FP64 combination
        elif h == 0:
            run = float(s)
        else:
            run = float(F(run + float(s)))            # stored running sum
    return run


def _case(rng, n, n_parts, scale_fn, extra_groups):
    values = scale_fn(rng, n).astype(F)
    classes = rng.integers(0, 8, n)
    parts_of = rng.integers(0, n_parts, n)
    own = [max([0] + [-(-int(np.sum((parts_of == h) & (classes == j))) // 4)
                      for j in range(8)]) for h in range(n_parts)]
    groups = [g + extra_groups for g in own]
    got = _kernel_sum(values, classes, parts_of, n_parts, groups)
    exact = math.fsum(float(v) for v in values)
    chain = max(groups) + 5 + max(0, n_parts - 2)
    bound = U32 * chain * float(np.sum(np.abs(values.astype(np.float64))))
    return abs(got - exact), bound, max(groups)


def test_quad4_summation_within_its_rounding_chain():
    rng = np.random.default_rng(20260)
    scales = [
        lambda r, n: r.normal(-8., 3., n),                          # log-slice like
        lambda r, n: -r.uniform(0., 1000., n),                      # with -1000 sentinels
        lambda r, n: np.where(r.random(n) < 0.5, 1e4, 1.) * r.normal(0., 1., n),
        lambda r, n: np.full(n, 1. + 2. ** -20) * np.where(np.arange(n) % 2, 1., -1.),
    ]
    worst = 0.
    for trial in range(300):
        n = int(rng.integers(0, 400))
        n_parts = int(rng.integers(1, 5))
        err, bound, g = _case(rng, n, n_parts, scales[trial % len(scales)],
                              int(rng.integers(0, 3)))
        assert err <= bound, (trial, n, n_parts, err, bound)
        if bound > 0:
            worst = max(worst, err / bound)
    print('largest error / chain bound: %.3g' % worst)


def test_chain_fits_the_threshold_budget():
    """G + 5 + max(0, P - 2) <= rows + 8 for rows >= G and P <= 4 parts."""
    for g in range(0, 200):
        for p in range(1, 5):
            assert g + 5 + max(0, p - 2) <= g + 8


def _sets_lane_sum(slots):
    """One lane of the frame-set kernel over its groups (four slots each,
    zero-column slots hold 0): group trees (v0 + v1) + (v2 + v3) go
    alternately into a0 and a1, then a0 + a1 -- float32."""
    g = slots.reshape(-1, 4).astype(F)
    a0, a1 = F(0.), F(0.)
    for i in range(g.shape[0]):
        t = F(F(g[i, 0] + g[i, 1]) + F(g[i, 2] + g[i, 3]))
        if i % 2 == 0:
            a0 = F(a0 + t)
        else:
            a1 = F(a1 + t)
    return F(a0 + a1)


def test_sets_summation_within_its_rounding_chain():
    """k_screen_sets: per part a frame's photons sit in some of its lane's
    4 G slots (G = the set's group count there); each value passes through at
    most ceil(G / 2) + 3 FP32 roundings per part, parts after the first add
    in FP64 (a stored running sum between parts when P > 2), so the chain
    ceil(Gmax / 2) + 3 + max(0, P - 2) fits rows + 8 with rows = ceil(Gmax / 2)
    (what the threshold is given for each frame)."""
    rng = np.random.default_rng(20261)
    scales = [
        lambda r, n: r.normal(-8., 3., n),
        lambda r, n: -r.uniform(0., 1000., n),
        lambda r, n: np.where(r.random(n) < 0.5, 1e4, 1.) * r.normal(0., 1., n),
        lambda r, n: np.full(n, 1. + 2. ** -20) * np.where(np.arange(n) % 2, 1., -1.),
    ]
    worst = 0.
    for trial in range(400):
        n = int(rng.integers(0, 500))
        n_parts = int(rng.integers(1, 5))
        values = scales[trial % len(scales)](rng, n).astype(F)
        part_of = rng.integers(0, n_parts, n)
        groups = []
        run = 0.
        for h in range(n_parts):
            v = values[part_of == h]
            g = -(-v.size // 4) + int(rng.integers(0, 4))      # the set may need more
            groups.append(g)
            slots = np.zeros(4 * g, dtype=F)
            slots[rng.permutation(4 * g)[:v.size]] = v
            s = float(_sets_lane_sum(slots))
            if h == n_parts - 1:
                run = run + s if h > 0 else s
            elif h == 0:
                run = float(F(s))
            else:
                run = float(F(run + s))
        exact = math.fsum(float(x) for x in values)
        gmax = max(groups) if groups else 0
        rows = -(-gmax // 2)
        chain = rows + 3 + max(0, n_parts - 2)
        assert chain <= rows + 8
        bound = U32 * chain * float(np.sum(np.abs(values.astype(np.float64))))
        assert abs(run - exact) <= bound, (trial, n, n_parts)
        if bound > 0:
            worst = max(worst, abs(run - exact) / bound)
    print('largest error / chain bound: %.3g' % worst)
