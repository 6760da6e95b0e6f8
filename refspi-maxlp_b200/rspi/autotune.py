"""Autotuner of the likelihood kernel's tiling.

For an E-step (its form, kernel, geometry and photon entries) the tuner
times the likelihood kernel on a sample of likelihood rows -- two tiles per
SM of the largest tile -- for every candidate tiling of that kernel, with
CUDA events on the launching stream, and keeps the fastest:

* ``sets`` and ``quad4`` (four rows per tile over column parts): warps per
  CTA and the number of column parts (the fewest that fit shared memory, or
  one more);
* ``stream`` / ``dynamic`` (the streaming and warp-per-frame kernels): rows
  per tile and warps per CTA.

The FP64-rescored argmax, maximum and log-sum-exp do not depend on the
tiling (every tiling keeps the screened FP32 values within the threshold's
error bound).  Results are cached in a JSON file keyed by GPU name, form,
kernel, detector geometry (slice row length, states), frame count and photon
entries, so later runs of the same geometry skip the search; the cache path
is ``$RSPI_AUTOTUNE_CACHE`` or ``~/.cache/rspi_autotune.json``.
"""
import json
import os

import torch

from .device import QUAD4_MAX_PARTS, quad4_parts

CACHE = os.environ.get('RSPI_AUTOTUNE_CACHE',
                       os.path.join(os.path.expanduser('~'), '.cache', 'rspi_autotune.json'))
TILES = (1, 2, 3, 4, 6, 8)
WARPS = (8, 16, 32)
WARPS_FOUR_ROW = (16, 24, 32)


def key(es):
    name = torch.cuda.get_device_name(es.device)
    ent = es.ll if es.form == 'fp64' else es.ll16
    return '%s|%s|%s|%d|%d|%d|%d' % (name, es.form, es.kernel, es.p_row, es.n_rows,
                                     es.ph.num_data, ent['total_rows'])


def candidates(es):
    """The tilings the tuner tries for ``es``: dicts of EStep.configure
    arguments."""
    if es.kernel in ('sets', 'quad4'):
        p0 = quad4_parts(es.p_row)[0]
        parts = [p for p in (p0, p0 + 1) if p <= QUAD4_MAX_PARTS]
        return [dict(warps=w, screen_parts=p) for p in parts for w in WARPS_FOUR_ROW]
    tmax = es.lib.rspi_loglike_max_tile(es.p_row, es.slice_code)
    return [dict(tile=t, warps=w) for t in TILES if t <= tmax for w in WARPS
            if es.form == 'screen' or not (t > 2 and w > 16)]


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(table):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        tmp = CACHE + '.tmp'
        with open(tmp, 'w') as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE)
    except OSError:
        pass


def _time(es, cfg, repeats):
    """Milliseconds per likelihood row of ``es`` under tiling ``cfg`` on a
    sample of rows (slices rebuilt in that tiling's layout)."""
    es.configure(**cfg)
    sms = torch.cuda.get_device_properties(es.device).multi_processor_count
    rows = min(es.n_rows, es.chunk_rows, sms * 2 * max(4, es.tile))
    es.rot_slices(0, rows)
    n = es.ph.num_data
    stream = torch.cuda.current_stream()
    es._loglike_launch(0, rows, es.lsl, n)          # warm-up
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(repeats):
        es._loglike_launch(0, rows, es.lsl, n)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / repeats / rows


def tune(es, repeats=3, use_cache=True, verbose=False):
    """Pick the fastest tiling for ``es`` and set it.  Returns (the chosen
    tiling, ms per row, all timings or None when taken from the cache).
    A model must have been sliced (``es.slices``) before: the timing reuses
    the E-step's slices of that model."""
    k = key(es)
    table = _load() if use_cache else {}
    if k in table:
        cfg = table[k]['config']
        es.configure(**cfg)
        return cfg, table[k]['ms_per_row'], None
    results = []
    for cfg in candidates(es):
        ms = _time(es, cfg, repeats)
        results.append((ms, cfg))
        if verbose:
            print('%s: %.5f us/row' % (cfg, ms * 1e3))
    ms, cfg = min(results, key=lambda r: r[0])
    es.configure(**cfg)
    es.ph.err.check('autotune')
    table[k] = {'config': cfg, 'ms_per_row': ms,
                'all': [[c, m] for m, c in results]}
    if use_cache:
        _save(table)
    return cfg, ms, results
