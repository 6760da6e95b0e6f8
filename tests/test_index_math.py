"""Host checks of kernel index arithmetic.  The pixel row/column (pixel_xy
in rspi_common.cuh): a float32 estimate of p / size, truncated, is within
one of the quotient for every pixel of the sizes the kernels accept, so one
correction step gives the exact row and column (exhaustive for small
sizes, sampled with the largest pixels up to size 46340).  The four-row
tile's column parts and gather bounds, and the rotation-major slice grid's
row coverage."""
import numpy as np
import pytest


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


def test_quad4_column_parts():
    """Column parts of the four-row frame-quad tile (k_screen_ll7): a
    multiple of 8 columns each, covering every likelihood column, the tile
    with its 8 zero columns within the kernel's dynamic shared memory, the
    pad q = part_w / 8 a 16-bit value, and the largest gather (q = part_w / 8,
    lane class 7) ending exactly at the tile's end."""
    from rspi.device import QUAD4_COLS, QUAD4_MAX_PARTS, QUAD4_SMEM, quad4_parts
    for p_row in range(64, 65536 + 1, 32):
        pz = p_row - 32
        if pz > QUAD4_MAX_PARTS * QUAD4_COLS:
            with pytest.raises(ValueError):
                quad4_parts(p_row)
            continue
        for forced in (None, 1, 2, 3, 4):
            try:
                parts, pw = quad4_parts(p_row, forced)
            except ValueError:
                assert forced is not None and -(-pz // forced) > QUAD4_COLS
                continue
            assert parts == (forced or parts) and 1 <= parts <= QUAD4_MAX_PARTS
            assert pw % 8 == 0 and parts * pw >= pz and pw >= 8
            assert (pw + 8) * 16 <= QUAD4_SMEM <= 227 * 1024 - 1024
            assert pw // 8 <= 0xffff
            last_byte = (pw // 8) * 128 + 16 * 7 + 16
            assert last_byte == (pw + 8) * 16
            if forced is None:   # the fewest parts that fit
                assert parts == 1 or -(-pz // (parts - 1)) > QUAD4_COLS


def test_rot_log_rotation_major_grid_covers_rows_once():
    """k_rot_log_js: CTA b takes rotation b mod R and states
    s_lo + 8 (b div R) .. + 7 clipped to the rows [row_begin, row_end); over
    all CTAs every row of the range is written exactly once and no other."""
    rng = np.random.default_rng(5)
    cases = [(405, 180, 0, 405 * 180), (7, 3, 0, 21), (20, 5, 13, 14), (20, 5, 13, 13 + 1),
             (1, 1, 0, 1), (50, 9, 100, 401)]
    for _ in range(40):
        s0, r = int(rng.integers(1, 60)), int(rng.integers(1, 40))
        a = int(rng.integers(0, s0 * r))
        cases.append((s0, r, a, int(rng.integers(a + 1, s0 * r + 1))))
    for n_states0, num_rot, rb, re in cases:
        s_lo, s_hi = rb // num_rot, (re - 1) // num_rot
        n_groups = (s_hi - s_lo) // 8 + 1
        seen = np.zeros(n_states0 * num_rot, dtype=np.int64)
        for b in range(n_groups * num_rot):
            j, first = b % num_rot, s_lo + (b // num_rot) * 8
            sb, se = first, first + 8
            while sb < se and sb * num_rot + j < rb:
                sb += 1
            while se > sb and (se - 1) * num_rot + j >= re:
                se -= 1
            for s in range(sb, se):
                assert s < n_states0
                seen[s * num_rot + j] += 1
        assert np.all(seen[rb:re] == 1) and seen[:rb].sum() == 0 and seen[re:].sum() == 0
