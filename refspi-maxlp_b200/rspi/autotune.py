"""Tile autotuner for the likelihood kernel (states per CTA x warps per CTA).

For a given E-step (its form, kernel, slice row length and entry stream) the
tuner times the E-step's likelihood kernel over a sample of likelihood rows
for every (states_per_tile, warps_per_cta) that fits in shared memory, with CUDA
events on the launching stream, and keeps the fastest.  Results are cached
in a JSON file keyed by device name, form, slice row length, frame count and
entry rows, so later runs of the same geometry skip the search.
"""
import json
import os

import torch


CACHE = os.environ.get('RSPI_AUTOTUNE_CACHE',
                       os.path.join(os.path.expanduser('~'), '.cache', 'rspi_autotune.json'))
TILES = (1, 2, 3, 4, 6, 8)
WARPS = (8, 16, 32)


def _key(es):
    name = torch.cuda.get_device_name(es.device)
    ent = es.ll if es.form == 'fp64' else es.ll16
    return '%s|%s|%s|%d|%d|%d' % (name, es.form, es.kernel, es.p_row, es.ph.num_data,
                                  ent['total_rows'])


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


def tune(es, sample_tiles=2, repeats=2, use_cache=True, verbose=False):
    """Pick (states_per_tile, warps) for ``es`` and set them on it.

    The sample covers ``sample_tiles`` tiles per SM of the largest tile size,
    so every candidate runs on the same rows.  Returns (tile, warps, ms
    per row) and a table of all timings."""
    key = _key(es)
    table = _load() if use_cache else {}
    if key in table:
        t, w = table[key]['tile'], table[key]['warps']
        es.tile, es.warps = t, w
        return (t, w, table[key]['ms_per_row']), None
    tmax = es.lib.rspi_loglike_max_tile(es.p_row, es.slice_code)
    if es.form == 'screen' and es.kernel == 'quad4':
        tiles = (4,)   # the four-row frame-quad kernel: warps per CTA only
    else:
        tiles = TILES
    cands = [(t, w) for t in tiles if t <= tmax for w in WARPS
             if es.form == 'screen' or not (t > 2 and w > 16)]
    sms = torch.cuda.get_device_properties(es.device).multi_processor_count
    rows = min(es.n_rows, es.chunk_rows, sms * sample_tiles * max(t for t, _ in cands))
    es.rot_slices(0, rows)
    n = es.ph.num_data
    stream = torch.cuda.current_stream()
    results = []
    for t, w in cands:
        def run():
            es.tile, es.warps = t, w
            es._loglike_launch(0, rows, es.lsl, n)
        run()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(repeats):
            run()
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / repeats / rows
        results.append((ms, t, w))
        if verbose:
            print('tile %d warps %2d: %.4f us/row' % (t, w, ms * 1e3))
    ms, t, w = min(results)
    es.tile, es.warps = t, w
    table[key] = {'tile': t, 'warps': w, 'ms_per_row': ms,
                  'all': [[r[1], r[2], r[0]] for r in results]}
    if use_cache:
        _save(table)
    return (t, w, ms), results
