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
