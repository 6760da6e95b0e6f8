"""Generate golden vectors by running the reference's own code on the CPU.

The reference (emc.py, maxLP.py, dset.py) is imported from the reference
tree unmodified.  CuPy/cupyx/h5py/mpi4py are replaced by the NumPy/SciPy
stand-ins in ``refshim/``; ``cupy.RawModule`` kernels execute the reference's
own kernels.cu compiled for the CPU by ``oracle/ref_cpu/build.py``.

Each case writes ``tests/golden/<name>.npz`` holding the inputs (photon
lists, config values, start model) and the reference outputs:

* Dataset attributes (ones_accum, multi_accum, mean_count, counts, powder);
* ``slice_gen_holo`` / ``slice_gen`` outputs for a few states and angles;
* for iterations 1 and 2 of ``EMC.run_iteration``: ``prob``, ``rmax`` and
  the model after the MaxLP M-step;
* MaxLPhaser pieces for a few pixels: photons, reference amplitudes,
  per-candidate rescale and log-likelihood;
* the posterior-weighted merge of the iteration-1 likelihoods through the
  reference's own merge_all and slice_merge kernels;
* the model refinement of MaxLPhaser._improve_model (support mask, one
  difference-map and one error-reduction step, the refined model) on the
  iteration-2 model, and in ``phase_a.npz`` on a compact 61x61 object.

Run from the repository root: ``python tests/golden/make_golden.py``.
Needs the reference tree (default ``/root/reference``).
"""
import contextlib
import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get('RSPI_REFERENCE_ROOT', '/root/reference')

sys.path.insert(0, os.path.join(REPO, 'refspi-maxlp_b200'))
from rspi import synth  # noqa: E402

CASES = {
    # name: generator + reconstruction settings
    'case_a': dict(size=21, num_data=40, mean_count=300., n_blobs=6, obj_radius=3.,
                   fluence_sigma=0.3, seed=11, num_rot=8, shiftx='-1 1 3',
                   shifty='-1 1 3', sphere_dia='2 3 2', need_scaling=True, bg=None,
                   model_seed=101),
    'case_b': dict(size=25, num_data=30, mean_count=400., n_blobs=8, obj_radius=4.,
                   fluence_sigma=0.5, seed=12, num_rot=6, shiftx='-1 1 2',
                   shifty='0 1 2', sphere_dia='2 4 3', need_scaling=False, bg=0.02,
                   model_seed=102),
}


def _write_inputs(tmp, name, c):
    data = synth.generate(c['size'], c['num_data'], c['mean_count'], c['n_blobs'],
                          c['obj_radius'], c['fluence_sigma'], (2., 4.), 1., seed=c['seed'])
    import h5py  # the stand-in
    path = os.path.join(tmp, 'photons.h5')
    with h5py.File(path, 'w') as f:
        f['num_pix'] = np.array([c['size'] ** 2])
        f['ones'] = data['ones']
        f['multi'] = data['multi']
        for key, lens in (('place_ones', data['ones']), ('place_multi', data['multi']),
                          ('count_multi', data['multi'])):
            bounds = np.concatenate([[0], np.cumsum(lens)])
            arr = np.empty(len(lens), dtype=object)
            for i in range(len(lens)):
                arr[i] = data[key][bounds[i]:bounds[i + 1]]
            f[key] = arr
        bg = None
        if c['bg'] is not None:
            rng = np.random.default_rng(c['seed'] + 1000)
            bg = c['bg'] * rng.random(c['size'] ** 2)
            f['bg'] = bg
    cfg = os.path.join(tmp, 'config.ini')
    with open(cfg, 'w') as f:
        f.write('[emc]\nsize = %d\nin_photons_file = photons.h5\noutput_folder = out/\n'
                'log_file = out/EMC.log\nneed_scaling = %s\nnum_rot = %d\nnum_modes = 1\n'
                'sphere_dia = %s\nshiftx = %s\nshifty = %s\n' %
                (c['size'], c['need_scaling'], c['num_rot'], c['sphere_dia'],
                 c['shiftx'], c['shifty']))
    os.makedirs(os.path.join(tmp, 'out'), exist_ok=True)
    return data, bg, cfg


def _merge_outputs(rec, prob, size, num_rot, ds):
    import cupy as cp   # the stand-in
    m = prob.max(0)
    e = np.exp(prob - m)
    post = e / e.sum(0)
    post = np.where(post >= ref_p_min(), post, 0.)
    n_rows, ndata = post.shape
    n0 = n_rows // num_rot
    scales = np.asarray(rec.scales, dtype='f8')
    num = np.zeros((n0, size * size)).view(cp.ndarray)
    den = np.zeros((n0, size * size)).view(cp.ndarray)
    mw = np.zeros(size * size).view(cp.ndarray)
    bsz = int(np.ceil(size / 32.))
    ones = np.ones(size * size)
    args = (np.asarray(ds.ones, dtype='i4'), np.asarray(ds.multi, dtype='i4'),
            np.asarray(ds.ones_accum, dtype='i8'), np.asarray(ds.multi_accum, dtype='i8'),
            np.asarray(ds.place_ones, dtype='i4'), np.asarray(ds.place_multi, dtype='i4'),
            np.asarray(ds.count_multi, dtype='i4'))
    for r in range(n_rows):
        w = float(post[r] @ scales)
        if w == 0.:
            continue
        s0, j = divmod(r, num_rot)
        view = np.zeros(size * size).view(cp.ndarray)
        rec.k_merge_all((int(np.ceil(ndata / 32.)),), (32,),
                        (np.ascontiguousarray(post[r]), ndata) + args + (view,))
        rec.k_slice_merge((bsz,) * 2, (32,) * 2, (view, j * np.pi / num_rot, size, num[s0], mw))
        rec.k_slice_merge((bsz,) * 2, (32,) * 2,
                          (np.ascontiguousarray(ones * w), j * np.pi / num_rot, size, den[s0], mw))
    return dict(merge_post=post, merge_num=np.asarray(num), merge_den=np.asarray(den))


def ref_p_min():
    import emc as ref_emc
    return ref_emc.P_MIN


def _phase_outputs(ph, fconv, sink):
    """The reference's ER / difference-map pieces on one model: the support
    mask of _improve_model (maxLP.py:292-298), one diffmap and one er step
    from the model itself (maxLP.py:282-289), and _improve_model's result
    (10 difference-map + 5 error-reduction iterations, maxLP.py:342-354)."""
    with contextlib.redirect_stdout(sink), contextlib.redirect_stderr(sink):
        fout = np.asarray(ph._improve_model(fconv.copy())).ravel()
        supp = np.asarray(ph.minvsuppmask).ravel()
        dm1 = np.asarray(ph.diffmap(fconv.copy(), fconv.copy())).ravel()
        er1 = np.asarray(ph.er(fconv.copy(), fconv.copy())).ravel()
    return dict(phase_in=fconv.copy(), phase_supp=supp, phase_dm1=dm1, phase_er1=er1,
                phase_out=fout, phase_invmask=np.asarray(ph.minvmask).ravel())


def run_phase_case(size=61, seed=13):
    """A model refinement case with a compact object: the Fourier transform
    of a blob density of radius 8 px plus noise, so the support is a proper
    subset of the image; run through a MaxLPhaser of the reference built on
    a two-frame photons file of that size."""
    rng = np.random.default_rng(seed)
    # densities of ~1e-2, so that the support threshold 1.2e-4 of
    # maxLP.py:296 cuts the smoothed object's tails
    obj = 1e-2 * synth.make_object(size, 10, 8., rng)
    f = synth.fourier(obj)
    f = f + 0.05 * np.abs(f).mean() * (rng.standard_normal(f.shape) +
                                       1j * rng.standard_normal(f.shape))
    with tempfile.TemporaryDirectory() as tmp:
        import h5py  # the stand-in
        path = os.path.join(tmp, 'photons.h5')
        with h5py.File(path, 'w') as fh:
            fh['num_pix'] = np.array([size ** 2])
            fh['ones'] = np.array([1, 1], dtype='i4')
            fh['multi'] = np.array([0, 0], dtype='i4')
            po = np.empty(2, dtype=object)
            po[0], po[1] = np.array([0], 'i4'), np.array([1], 'i4')
            pm = np.empty(2, dtype=object)
            pm[0], pm[1] = np.zeros(0, 'i4'), np.zeros(0, 'i4')
            fh['place_ones'] = po
            fh['place_multi'] = pm
            fh['count_multi'] = pm
        cwd = os.getcwd()
        os.chdir(REF)
        try:
            import maxLP as ref_maxlp
            sink = io.StringIO()
            with contextlib.redirect_stdout(sink), contextlib.redirect_stderr(sink):
                ph = ref_maxlp.MaxLPhaser(path, size=size)
            out = _phase_outputs(ph, f.ravel().astype(np.complex128), sink)
        finally:
            os.chdir(cwd)
    out['size'] = np.array(size)
    return out


def run_case(name, c):
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        data, bg, cfg = _write_inputs(tmp, name, c)
        model0 = synth.initial_model(c['size'], c['model_seed'])
        cwd = os.getcwd()
        os.chdir(REF)           # maxLP.py opens 'kernels.cu' by relative path
        try:
            import emc as ref_emc
            np.random.seed(0)
            sink = io.StringIO()
            with contextlib.redirect_stdout(sink), contextlib.redirect_stderr(sink):
                rec = ref_emc.EMC(cfg, num_streams=4)
            rec.model = model0.copy()
            ds = rec.dset
            out.update(ds_ones_accum=np.asarray(ds.ones_accum), ds_multi_accum=np.asarray(ds.multi_accum),
                       ds_mean_count=np.array(ds.mean_count), ds_powder=np.asarray(rec.powder),
                       ds_bg=np.asarray(ds.bg))
            if c['need_scaling']:
                out['ds_counts'] = np.asarray(ds.counts)
            out['scales'] = np.asarray(rec.scales, dtype='f8')

            # single-kernel goldens
            size = c['size']
            bsz = int(np.ceil(size / 32.))
            holo, rot = [], []
            for r in range(min(3, rec.shiftx.size)):
                v = np.zeros(size ** 2).view(type(np.asarray(rec.powder)))
                rec.k_slice_gen_holo((bsz,) * 2, (32,) * 2,
                                     (np.ascontiguousarray(model0), rec.shiftx[r], rec.shifty[r],
                                      rec.sphere_dia[r], 1., 1., size, rec.dset.bg, 0, v))
                holo.append(np.array(v))
                for j in (0, 1, c['num_rot'] - 1):
                    lv = np.zeros(size ** 2).view(type(v))
                    rec.k_slice_gen((bsz,) * 2, (32,) * 2,
                                    (v, j * np.pi / rec.num_rot, 1., size, rec.dset.bg, 1, lv))
                    rot.append(np.array(lv))
            out['holo'] = np.array(holo)
            out['rotlog'] = np.array(rot)

            for it in (1, 2):
                with contextlib.redirect_stdout(sink), contextlib.redirect_stderr(sink):
                    model_in = np.array(rec.model)
                    rec.run_iteration(it)
                out['model_in_%d' % it] = model_in
                out['prob_%d' % it] = np.array(rec.prob, copy=True)
                out['rmax_%d' % it] = np.array(rec.rmax, copy=True)
                out['model_out_%d' % it] = np.array(rec.model)
                sx, sy, dia, ang = rec._unravel_rmax(rec.rmax)
                out['unravel_%d' % it] = np.stack([np.asarray(sx), np.asarray(sy),
                                                   np.asarray(dia), np.asarray(ang)])
                resc = [line for line in sink.getvalue().splitlines()
                        if line.startswith('Estimated rescale:')]
                out['rescale_%d' % it] = np.array(float(resc[-1].split(':')[1]))

            # posterior-weighted merge with the reference's own merge_all and
            # slice_merge kernels (kernels.cu:84-152, loaded by emc.py:104,107
            # but not launched on its run path) on the iteration-1
            # likelihoods: posteriors normalised per frame, those below P_MIN
            # dropped, the data-space sums of each row back-rotated into its
            # (shift, diameter) state, and the weights sum_d P scale_d likewise
            out.update(_merge_outputs(rec, out['prob_1'], size, c['num_rot'], ds))

            # phaser pieces on the state left by iteration 2
            import cupy as cp   # the stand-in
            ph = rec.phaser
            pix = np.where(np.asarray(ph.mask))[0]
            pick = pix[np.linspace(0, pix.size - 1, 5).astype(int)]
            pick = np.concatenate([pick, pix[np.argsort(-np.asarray(rec.powder)[pix])[:3]]])
            k_l, fr_l, lq_l, rs_l, cand_l = [], [], [], [], []
            for t in pick:
                const = ph.get_pixel_constants(int(t))
                f_t = complex(out['model_in_2'][t])
                cand = f_t + np.asarray(ph.pattern) * (abs(f_t) / 4.)
                k_l.append(np.asarray(const['k_d']).ravel())
                fr_l.append(np.asarray(const['fref_d']))
                rs_l.append(np.asarray(ph.get_rescale_pixel(cp.asarray(cand), int(t), const)))
                lq_l.append(np.asarray(ph.get_logq_pixel(cp.asarray(cand), int(t),
                                                         rescale=None, const=const)))
                cand_l.append(cand)
            out.update(ph_pixels=pick, ph_k=np.array(k_l), ph_fref=np.array(fr_l),
                       ph_rescale=np.array(rs_l), ph_logq=np.array(lq_l), ph_cand=np.array(cand_l),
                       ph_shifts=np.asarray(ph.shifts), ph_diams=np.asarray(ph.diams),
                       ph_ang=np.asarray(ph.ang))
            # model refinement (maxLP.py:271-354) on the iteration-2 model
            out.update(_phase_outputs(ph, np.asarray(out['model_out_2']).ravel(), sink))
        finally:
            os.chdir(cwd)
    out.update(model0=model0, size=np.array(c['size']), num_rot=np.array(c['num_rot']),
               shiftx=np.array(c['shiftx']), shifty=np.array(c['shifty']),
               sphere_dia=np.array(c['sphere_dia']), need_scaling=np.array(c['need_scaling']),
               ones=data['ones'], multi=data['multi'], place_ones=data['place_ones'],
               place_multi=data['place_multi'], count_multi=data['count_multi'])
    if bg is not None:
        out['bg'] = bg
    return out


def main():
    sys.path.insert(0, os.path.join(REPO, 'oracle', 'ref_cpu'))
    import build as ref_build
    if ref_build.build(REF, quiet=True) is None:
        raise SystemExit('reference tree not found at %s' % REF)
    sys.path.insert(0, os.path.join(HERE, 'refshim'))
    sys.path.insert(1, REF)
    for name, c in CASES.items():
        res = run_case(name, c)
        path = os.path.join(HERE, name + '.npz')
        np.savez_compressed(path, **res)
        print(name, '->', path, '%.1f KB' % (os.path.getsize(path) / 1024))
    path = os.path.join(HERE, 'phase_a.npz')
    np.savez_compressed(path, **run_phase_case())
    print('phase_a ->', path, '%.1f KB' % (os.path.getsize(path) / 1024))


if __name__ == '__main__':
    main()
