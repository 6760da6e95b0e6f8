"""Host check of the kernels' pixel row/column arithmetic (pixel_xy in
rspi_common.cuh): a float32 estimate of p / size, truncated, is within one
of the quotient for every pixel of the sizes the kernels accept, so one
correction step gives the exact row and column.  Exhaustive for small
sizes, sampled (with the largest pixels) up to size 46340."""
import numpy as np


def _pixel_xy(p, size):
    inv = np.float32(1.) / np.float32(size)
    q = (p.astype(np.float32) * inv).astype(np.int64)   # truncation, as (int)
    r = p - q * size
    low, high = r < 0, r >= size
    q = q - low + high
    r = r + size * low - size * high
    return q, r


def _check(p, size):
    q, r = _pixel_xy(p, size)
    assert np.array_equal(q, p // size) and np.array_equal(r, p % size), size
    # the estimate itself never misses by more than one
    est = (p.astype(np.float32) * (np.float32(1.) / np.float32(size))).astype(np.int64)
    assert np.all(np.abs(est - p // size) <= 1), size


def test_pixel_xy_exhaustive_small_sizes():
    for size in list(range(2, 130)) + [185, 255, 256, 511, 512]:
        _check(np.arange(size * size, dtype=np.int64), size)


def test_pixel_xy_sampled_large_sizes():
    rng = np.random.default_rng(0)
    for size in (1000, 4097, 16384, 30001, 46339, 46340):
        n = size * size
        p = np.concatenate([rng.integers(0, n, 2_000_000), np.arange(n - 100_000, n),
                            np.arange(0, n, size), np.arange(size - 1, n, size)])
        _check(p.astype(np.int64), size)
