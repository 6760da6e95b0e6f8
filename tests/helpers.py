"""Shared helpers for the test-suite: golden cases, oracle set-ups and small
random datasets (all seeded)."""
import os

import numpy as np

from conftest import GOLDEN
from oracle import emc_oracle as E

GOLDEN_CASES = ('case_a', 'case_b')


def load_golden(name):
    g = np.load(os.path.join(GOLDEN, name + '.npz'))
    return {k: g[k] for k in g.files}


def golden_dataset(g):
    size = int(g['size'])
    bg = g.get('bg')
    ds = E.parse_photons(g['ones'], g['multi'], g['place_ones'], g['place_multi'],
                         g['count_multi'], size * size, bool(g['need_scaling']), bg)
    return ds


def golden_states(g):
    return E.generate_states(E.parse_triple(str(g['shiftx'])), E.parse_triple(str(g['shifty'])),
                             E.parse_triple(str(g['sphere_dia'])))


def write_case(tmpdir, g=None, data=None, size=None, num_rot=None, shiftx=None, shifty=None,
               sphere_dia=None, need_scaling=None, extra=''):
    """Write photons + config.ini for EMC; returns the config path."""
    from rspi.photonfile import write_photons
    if g is not None:
        size = int(g['size'])
        data = dict(num_pix=np.array([size * size]), ones=g['ones'], multi=g['multi'],
                    place_ones=g['place_ones'], place_multi=g['place_multi'],
                    count_multi=g['count_multi'])
        if 'bg' in g:
            data['bg'] = g['bg']
        num_rot = int(g['num_rot'])
        shiftx, shifty, sphere_dia = str(g['shiftx']), str(g['shifty']), str(g['sphere_dia'])
        need_scaling = bool(g['need_scaling'])
    os.makedirs(os.path.join(tmpdir, 'out'), exist_ok=True)
    write_photons(os.path.join(tmpdir, 'photons.npz'), data)
    cfg = os.path.join(tmpdir, 'config.ini')
    with open(cfg, 'w') as f:
        f.write('[emc]\nsize = %d\nin_photons_file = photons.npz\noutput_folder = out/\n'
                'log_file = out/EMC.log\nneed_scaling = %s\nnum_rot = %d\nnum_modes = 1\n'
                'sphere_dia = %s\nshiftx = %s\nshifty = %s\n%s' %
                (size, need_scaling, num_rot, sphere_dia, shiftx, shifty, extra))
    return cfg


def random_photons(size, n, mean, seed, empty_frames=(), masked_frames=(), heavy=None):
    """Random sparse photon lists with a few edge cases: empty frames, frames
    with photons only outside the likelihood mask, and optionally a heavy
    frame with many multi-photon pixels."""
    rng = np.random.default_rng(seed)
    npix = size * size
    _, probmask = E.generate_masks(size)
    outside = np.flatnonzero(probmask >= 1)
    ones, multi, po, pm, cm = [], [], [], [], []
    for d in range(n):
        lam = np.full(npix, mean / npix)
        if heavy is not None and d == heavy:
            lam = lam * 50
        k = rng.poisson(lam)
        if d in empty_frames:
            k[:] = 0
        if d in masked_frames:
            k[:] = 0
            k[rng.choice(outside, size=min(5, outside.size), replace=False)] = 2
        o = np.flatnonzero(k == 1).astype('i4')
        m = np.flatnonzero(k > 1).astype('i4')
        ones.append(o.size)
        multi.append(m.size)
        po.append(o)
        pm.append(m)
        cm.append(k[m].astype('i4'))
    cat = lambda a: np.concatenate(a).astype('i4') if a else np.zeros(0, 'i4')  # noqa: E731
    return dict(num_pix=np.array([npix]), ones=np.array(ones, 'i4'), multi=np.array(multi, 'i4'),
                place_ones=cat(po), place_multi=cat(pm), count_multi=cat(cm))
