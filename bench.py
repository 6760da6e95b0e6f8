#!/usr/bin/env python
"""Benchmark of the RefSPI-MaxLP reconstruction hot path on B200.

Workload (default): the production-shape plain-method configuration --
185x185 detector, 20,000 synthetic frames at 2,000 photons/frame,
180 rotations x 9x9 shifts x 5 diameters = 72,900 states per frame.  One
step = one EMC iteration: likelihood of every frame in every state, per-frame
max/argmax/log-sum-exp, and the MaxLP M-step over every phaser pixel.

Our arm prints one JSON line with the metric (frame-state evaluations per
second of whole iterations, and s/iteration), measured with CUDA events on
the launching stream over K timed steps after W warm-up steps (inputs are
larger than L2), plus ``e2e`` through ``EMC.run_iteration`` (model copied
host->device and model + argmax copied back every step), the roofline of the
dominant kernel from live CUDA events, sampled SM clocks and a CPU baseline
(the FP64 NumPy oracle on the host cores, bounded sample, extrapolated).

``--impl reference`` times the reference's CPU equations (the FP64 oracle,
the reference having no CPU path of its own) on all host cores on a bounded
sample of the same workload and prints the same metric; its
``reference_gpu`` field adds the reference's own kernels.cu on the same GPU
(built from the reference sources, emc.py's and maxLP.py's loops replayed
with torch in place of CuPy), also on a bounded sample.

``--config 3`` evaluates the adjoint instead (NLL + gradient throughput,
L-BFGS against the polar grid search on NLL and FRC); ``--config 4`` and
``--config 5`` run the multi-mode and the dense high-fluence workloads.

Multi-GPU (torchrun, one process per GPU, NCCL): one job whose frames are
split over the ranks -- each rank draws its own ``--frames`` frames of the
same object (weak scaling), the E-step needs no exchange, the M-step sums
the pixel histograms over ranks and splits the pattern search by pixels
(rspi/shard.py); value = all ranks' frames x states / the slowest rank's
time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, 'refspi-maxlp_b200')
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = 'frame-state evaluations/s (EMC iteration: E-step + MaxLP M-step)'
UNIT = 'frame*state/s'
PEAKS_FALLBACK = {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}


# ---------------------------------------------------------------------------
def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--config', type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help='3: the adjoint evaluation on config-2 data (NLL, FRC, L-BFGS vs grid)')
    ap.add_argument('--frames', type=int, default=None, help='override frame count (testing)')
    ap.add_argument('--form', default=None, choices=['fp64', 'screen', 'dense'],
                    help='likelihood form (default: dense for config 5, screen otherwise)')
    ap.add_argument('--kernel', default=None, choices=['stream', 'quad4', 'sets', 'dynamic'],
                    help='likelihood kernel (default: the EStep default of the form)')
    ap.add_argument('--warps', type=int, default=None,
                    help='warps per CTA of the likelihood kernel (default: the EStep default, 32)')
    ap.add_argument('--screen-delta', type=float, default=None,
                    help='FP64 rescoring window in nats (EMC default 0: the argmax candidates)')
    ap.add_argument('--mstep', default=None, choices=['pattern', 'grid', 'lbfgs', 'grid+lbfgs'],
                    help='M-step: the MaxLP pattern search (default), or the pixel-NLL grid / '
                         'L-BFGS through the adjoint after its ring pass')
    ap.add_argument('--slice-math', default=None, choices=['fp64', 'fp32'],
                    help='arithmetic of the frame-set kernel\'s log-slices')
    ap.add_argument('--set-order', default=None, choices=['grouped', 'rank'],
                    help='frames of the frame-set kernel\'s quarter warps: grouped by class '
                         'totals (default) or in rank order')
    ap.add_argument('--merge', action='store_true',
                    help='each iteration also merges the posterior-weighted intensities '
                         '(row a10; rescoring window 20 nats)')
    ap.add_argument('--no-autotune', action='store_true',
                    help='keep the likelihood kernel\'s default tiling')
    ap.add_argument('--no-phaser-screen', action='store_true',
                    help='pattern search: every candidate in FP64 (no FP32 screening pass)')
    ap.add_argument('--slice-gb', type=float, default=8.,
                    help='largest rotated-slice chunk (GB); smaller values give more launches')
    ap.add_argument('--no-plain', action='store_true',
                    help='skip timing the plain form (FP64, dynamic kernel) for comparison')
    ap.add_argument('--cpu-seconds', type=float, default=20.,
                    help='target CPU time of the bounded oracle sample')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-clocks', action='store_true', help='do not sample nvidia-smi clocks')
    ap.add_argument('--no-ref-gpu', action='store_true',
                    help='reference arm: skip timing the reference kernels on the GPU')
    args = ap.parse_args()
    if args.form is None:
        from rspi import synth
        args.form = 'dense' if synth.CONFIGS.get(args.config, {}).get('dense') else 'screen'
    return args


def max_over_ranks(x, device):
    """The largest of ``x`` over all ranks of the initialised process group
    (``x`` itself without one): the job's time is its slowest rank's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    try:
        with open(os.path.join(REPO, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return {'hbm_gbs': float(p['hbm_gbs']), 'bf16_tflops': float(p['bf16_tflops']),
                'source': 'measured'}
    except Exception:
        return dict(PEAKS_FALLBACK, source='fallback')


def workload(cfg_id, frames):
    from rspi import synth
    c = synth.CONFIGS[cfg_id]
    n = c['num_data'] if frames is None else frames
    r = c['recon']
    nsx = int(r['shiftx'].split()[2])
    nsy = int(r['shifty'].split()[2])
    nd = int(r['sphere_dia'].split()[2])
    nm = int(r.get('num_modes', 1))
    return dict(cfg=c, n=n, size=c['size'], num_rot=r['num_rot'], n_states0=nsx * nsy * nd,
                n_modes=nm, n_states=nsx * nsy * nd * r['num_rot'] * nm, recon=r)


def workload_name(cfg_id, w):
    return ('config%d: %dx%d detector, %d frames, %d rotations x %d (shift,dia) states x %d '
            'mode(s) = %d states/frame, 1 EMC iteration per step' %
            (cfg_id, w['size'], w['size'], w['n'], w['num_rot'], w['n_states0'], w['n_modes'],
             w['n_states']))


def generate_data(cfg_id, w, device='cpu', rank=0):
    """The configuration's seeded synthetic photons (``w['n']`` frames;
    rank r > 0 of a multi-GPU job draws its own frames of the same object)."""
    from rspi import synth
    c = w['cfg']
    return synth.generate(c['size'], w['n'], c['mean_count'], c['n_blobs'], c['obj_radius'],
                          c['fluence_sigma'], c['dia'], c['shift_max'], seed=20260000 + cfg_id,
                          device=device, frame_seed=None if rank == 0 else 7919 * rank,
                          **synth.config_extras(cfg_id))


def start_model(cfg_id, w):
    """Seeded start model, one random image per mode (flattened)."""
    from rspi import synth
    return np.concatenate([synth.initial_model(w['size'], 20260100 + cfg_id + 1000 * m)
                           for m in range(w['n_modes'])])


def dram_traffic(args, w, es, rows_per_launch):
    """DRAM bytes (read + write) of one likelihood launch from the committed
    ncu capture of the same workload (form, configuration, frames, rows per
    launch), or None when no capture matches."""
    path = os.path.join(REPO, 'profiles', 'k_screen_config2_dram.json')
    try:
        with open(path) as f:
            caps = json.load(f)['captures']
    except (OSError, ValueError, KeyError):
        return None
    kern = es.kernel
    for c in caps:
        if (c['form'] == es.form and c.get('kernel', 'stream') == kern and
                c['config'] == args.config and c['frames'] == w['n'] and
                c['rows_per_launch'] == int(round(rows_per_launch))):
            return float(c['dram_bytes_read'] + c['dram_bytes_write'])
    return None


def roofline_blocks(args, w, es, ll_ms, ll_launches, ms, clk, pk, sm_count):
    """Roofline of the dominant kernel (the likelihood kernel, row a7) from
    its live CUDA-event time: HBM bytes for the sparse forms, tensor FLOPs
    for the dense form; plus the on-chip gather roofline of the sparse
    forms.  Returns (roofline, gather roofline or None, rows per launch)."""
    rows_per_launch = es.n_rows / max(1, ll_launches)
    ll_launch_ms = ll_ms / max(1, ll_launches)
    common = {'launch_ms': ll_launch_ms, 'launches_per_step': ll_launches,
              'share_of_step': ll_ms / ms}
    if es.form == 'dense':
        if es.dense_gemm == 'i8':
            # 2 int8 ops per (frame, pixel, row) for each of the 4 L digits;
            # the int8 dense tensor rate is twice the BF16 one
            flops = 2. * w['n'] * es.k_pad * rows_per_launch * 4
            peak, unit = 2. * pk['bf16_tflops'], 'TOP/s'
            src = pk['source'] + ' (2 x the cuBLAS bf16 GEMM burst: int8 runs at twice bf16)'
            a_bytes, name = w['n'] * es.k_pad, 'k_dense_ll<i8> (tcgen05 int8 GEMM, row a7)'
        else:
            # 2 FLOPs per (frame, pixel, row) for each count digit x (hi, lo)
            flops = 2. * w['n'] * es.k_pad * rows_per_launch * es.n_digits * 2
            peak, unit = pk['bf16_tflops'], 'TFLOP/s'
            src = pk['source'] + ' (cuBLAS bf16 GEMM, burst)'
            a_bytes = w['n'] * es.k_pad * 2 * es.n_digits
            name = 'k_dense_ll<bf16> (tcgen05 BF16 GEMM, row a7)'
        achieved = flops / (ll_launch_ms * 1e-3) / 1e12
        bytes_alg = a_bytes + rows_per_launch * es.k_pad * 4 + rows_per_launch * w['n'] * 4
        roof = dict({'kernel': name, 'bound': 'tensor', 'achieved': achieved, 'peak': peak,
                     'unit': unit, 'frac': achieved / peak, 'traffic': None, 'peak_source': src,
                     'flops_per_launch': flops, 'algorithmic_bytes_per_launch': bytes_alg}, **common)
        return roof, None, rows_per_launch
    total_rows = es.ll16['total_rows'] if es.form == 'screen' else es.ll['total_rows']
    esz = {0: 4, 1: 8}[es.slice_code]
    osz = 4 if es.prob_code == 0 else 8
    # algorithmic bytes per launch = its slices in + its LL rows out + the
    # packed photon entries once
    ent_bytes = total_rows * 32 * (2 if es.form == 'screen' else 4)
    alg_bytes = rows_per_launch * (es.p_row * esz + w['n'] * osz) + ent_bytes + 8 * w['n']
    achieved = alg_bytes / (ll_launch_ms * 1e-3) / 1e9
    # on-chip gather roofline.  Screened form: one shared-memory value per
    # photon (count-expanded, on likelihood pixels) per likelihood row; the
    # padded entry slots the kernel gathers (its conflict-free layout) as
    # slots_frac.  FP64 form: one value per (pixel, count) entry slot.
    slots = total_rows * 32
    if es.wide is not None and 'total_groups' in es.wide:
        slots = es.wide['total_groups'] * 128
    if es.form == 'screen':
        work = int(es.ll['frame_sel_photons'].sum().item())
    else:
        work = total_rows * 32
    gathers = rows_per_launch * work
    clk_mhz = (clk or {}).get('sm_mhz') or 1965.
    # values a shared-memory wavefront (128 B per clock) carries
    lanes = {0: 32, 1: 16}[es.slice_code]
    gather_peak = sm_count * lanes * clk_mhz * 1e6
    gather_rate = gathers / (ll_launch_ms * 1e-3)
    slots_rate = rows_per_launch * slots / (ll_launch_ms * 1e-3)
    names = {'stream': 'k_ll_stream<FormScreen>', 'quad4': 'k_screen_ll7',
             'sets': 'k_screen_sets'}
    roof = dict({'kernel': ('%s (FP32 screening likelihood, row a7)' %
                            names.get(es.kernel, es.kernel)
                            if es.form == 'screen' else 'k_ll_stream / k_loglike (FP64 likelihood, row a7)'),
                 'bound': 'hbm', 'achieved': achieved, 'peak': pk['hbm_gbs'], 'unit': 'GB/s',
                 'frac': achieved / pk['hbm_gbs'],
                 'traffic': dram_traffic(args, w, es, rows_per_launch),
                 'peak_source': pk['source'] + ' (HBM copy)'}, **common)
    gather = {'achieved': gather_rate, 'peak': gather_peak, 'unit': 'values/s',
              'frac': gather_rate / gather_peak, 'slots_frac': slots_rate / gather_peak,
              'slot_efficiency': work / max(1, slots),
              'note': ('%s per likelihood row against the shared-memory value rate %d SMs x '
                       '%d values/clk x %.0f MHz; slots_frac: the entry slots the kernel '
                       'gathers, padding included'
                       % ('photons' if es.form == 'screen' else 'entry slots', sm_count, lanes,
                          clk_mhz))}
    return roof, gather, rows_per_launch


def write_inputs(tmp, w, data, form, slice_gb=8., screen_delta=None, kernel=None, mstep=None,
                 autotune=True, rank=None, slice_math=None, merge=False, set_order=None):
    from rspi.photonfile import write_photons
    os.makedirs(os.path.join(tmp, 'out'), exist_ok=True)
    name = 'photons.npz' if rank is None else 'photons_%d.npz' % rank
    write_photons(os.path.join(tmp, name), data)
    cfg = os.path.join(tmp, 'config.ini')
    r = w['recon']
    with open(cfg, 'w') as f:
        f.write('[emc]\nsize = %d\nin_photons_file = %s\noutput_folder = out/\n'
                'log_file = out/EMC.log\nneed_scaling = True\nnum_rot = %d\nnum_modes = %d\n'
                'sphere_dia = %s\nshiftx = %s\nshifty = %s\nform = %s\nslice_budget_gb = %g\n' %
                (w['size'], 'photons.npz' if rank is None else 'photons_{rank}.npz',
                 r['num_rot'], w['n_modes'], r['sphere_dia'], r['shiftx'], r['shifty'],
                 form, slice_gb))
        if screen_delta is not None:
            f.write('screen_delta = %r\n' % float(screen_delta))
        if kernel:
            f.write('kernel = %s\n' % kernel)
        if mstep:
            f.write('mstep = %s\n' % mstep)
        if slice_math:
            f.write('slice_math = %s\n' % slice_math)
        if merge:
            f.write('merge = true\n')
        if set_order:
            f.write('set_order = %s\n' % set_order)
        f.write('autotune = %s\n' % bool(autotune))
    return cfg


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix='.csv')
            os.close(fd)
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.QUERY,
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(',')]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace('.', '').isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == 'active'})
        return {'sm_mhz': float(np.median(sm)) if sm else None,
                'sm_max_mhz': max(smax) if smax else None, 'reasons': reasons,
                'samples': len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle on the host cores, bounded sample
# ---------------------------------------------------------------------------
def _cpu_worker_init():
    os.environ['OMP_NUM_THREADS'] = '1'
    os.environ['OPENBLAS_NUM_THREADS'] = '1'
    os.environ['MKL_NUM_THREADS'] = '1'
    for p in (REPO, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)


def _cpu_estep_task(args):
    """Rotated log-slices of one state (all rotations) + their likelihood
    against a frame subset; returns (slice seconds, likelihood seconds)."""
    model, sx, sy, dia, size, num_rot, bg, kmat_sub = args
    from oracle import emc_oracle as E
    _, pm = E.generate_masks(size)
    sel = pm < 1
    t0 = time.perf_counter()
    lsl = E.log_slices_for_state(model, sx, sy, dia, size, bg, num_rot, sel)
    t1 = time.perf_counter()
    np.asarray(kmat_sub @ lsl.T)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1


def _cpu_maxlp_task(args):
    """Pattern search of one pixel over a frame subset (rescale given)."""
    f_t, k_d, fref_d, rescale = args
    from oracle import maxlp_oracle as M
    pat = M.gen_pattern(8)
    t0 = time.perf_counter()
    M.run_pixel_pattern(f_t, k_d, fref_d, pat, rescale, 10)
    return time.perf_counter() - t0


def _baseline_inputs(w, data):
    """Photon lists and per-frame values the CPU sample works on."""
    from oracle import emc_oracle as E
    from oracle import maxlp_oracle as M
    from rspi import geometry
    size, n = w['size'], w['n']
    ds = E.parse_photons(data['ones'], data['multi'], data['place_ones'], data['place_multi'],
                         data['count_multi'], size * size, True)
    _, pm = E.generate_masks(size)
    nf = min(n, 500)
    r = w['recon']
    sx, sy, dia, _ = geometry.state_grid(geometry.parse_triple(r['shiftx']),
                                         geometry.parse_triple(r['shifty']),
                                         geometry.parse_triple(r['sphere_dia']))
    kmat = E.sparse_frames(ds)
    qx, qy, qrad, mask, rmask = M.get_qvals(size)
    rng = np.random.default_rng(0)
    ang = rng.integers(0, w['num_rot'], n) * np.pi / w['num_rot']
    shifts = np.stack([rng.choice(np.unique(sx), n), rng.choice(np.unique(sy), n)], 1)
    diams = rng.choice(np.unique(dia), n)
    return dict(ds=ds, nf=nf, kmat_sel=E.sparse_frames(ds, pm < 1)[:nf], sx=sx, sy=sy, dia=dia,
                kmat=kmat, q=(qx, qy, qrad), main=np.flatnonzero(mask),
                n_phaser=int(rmask.sum() + mask.sum()), ang=ang, shifts=shifts, diams=diams)


def _baseline_sample(w, inp, model, pool, cores, n_est, npx):
    """Seconds per iteration of the FP64 oracle on ``cores`` workers,
    extrapolated from a bounded sample.

    E-step: ``n_est`` (shift, diameter) states x all rotations, likelihood
    against the first ``nf`` frames -> per-slice-row and per-(row, frame)
    costs, scaled to all rows and frames.  M-step: ``npx`` pixels over
    ``nf2`` frames -> per (pixel, frame) cost, scaled to every phaser pixel
    (ring + main pass) and all frames.  Linear extrapolation, stated in
    ``sample``.
    """
    from oracle import maxlp_oracle as M
    size, num_rot, n = w['size'], w['num_rot'], w['n']
    nf, sx, sy, dia = inp['nf'], inp['sx'], inp['sy'], inp['dia']
    picks = np.linspace(0, sx.size - 1, n_est).astype(int)
    t_wall0 = time.perf_counter()
    est = pool.map(_cpu_estep_task, [(model, sx[i], sy[i], dia[i], size, num_rot,
                                      inp['ds']['bg'], inp['kmat_sel']) for i in picks])
    t_slice_row = np.mean([a for a, _ in est]) / num_rot
    t_ll_cell = np.mean([b for _, b in est]) / (num_rot * nf)
    qx, qy, qrad = inp['q']
    main = inp['main']
    nf2 = min(n, 2000)
    tasks = []
    for t in main[np.linspace(0, main.size - 1, npx).astype(int)]:
        k = M.photons_pixel(inp['kmat'], inp['ang'], int(t), size, qx, qy)[:nf2]
        fr = M.fref_pixel(int(t), qx, qy, qrad, inp['diams'], inp['shifts'])[:nf2]
        tasks.append((complex(model[t]), k, fr, 1.0))
    mt = pool.map(_cpu_maxlp_task, tasks)
    wall = time.perf_counter() - t_wall0
    t_px_frame = np.mean(mt) / nf2
    rows = w['n_states']
    serial = rows * t_slice_row + rows * n * t_ll_cell + inp['n_phaser'] * n * t_px_frame
    per_iter = serial / cores
    return dict(s_per_iteration=per_iter, cores=cores, wall_s=wall,
                sample=('FP64 NumPy oracle, %d workers: E-step %d of %d (shift,dia) states x %d '
                        'rotations vs %d of %d frames, M-step %d pixels x %d frames; linear '
                        'extrapolation to %d rows x %d frames and %d phaser pixels, divided by '
                        'the worker count' % (cores, n_est, w['n_states0'], num_rot, nf, n, npx,
                                              nf2, rows, n, inp['n_phaser'])))


def _baseline_pool(cores):
    import multiprocessing as mp
    return mp.get_context('spawn').Pool(cores, initializer=_cpu_worker_init)


def cpu_baseline(w, data, model, target_s):
    """Extrapolated seconds per iteration of the FP64 oracle on all host
    cores (one bounded sample; see ``_baseline_sample``)."""
    cores = os.cpu_count() or 1
    inp = _baseline_inputs(w, data)
    with _baseline_pool(cores) as pool:
        return _baseline_sample(w, inp, model, pool, cores, max(1, min(cores, 8)), max(cores, 8))


# ---------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return 0
    w = workload(args.config, args.frames)
    data = generate_data(args.config, w)
    model = start_model(args.config, w)[:w['size'] ** 2]
    cores = os.cpu_count() or 1
    inp = _baseline_inputs(w, data)
    times = []
    base = None
    with _baseline_pool(cores) as pool:
        for _ in range(args.warmup):
            # untimed: one state and one pixel load the oracle in every worker
            _baseline_sample(w, inp, model, pool, cores, 1, 1)
        for _ in range(args.steps):
            base = _baseline_sample(w, inp, model, pool, cores, max(1, min(cores, 8)),
                                    max(cores, 8))
            times.append(base['s_per_iteration'])
    t = float(np.mean(times))
    v = w['n'] * w['n_states'] / t
    out = {'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': UNIT,
           'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
           'ms_per_step': t * 1e3, 's_per_iteration': t, 'higher_is_better': True,
           'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
           'config': {'workload': workload_name(args.config, w), 'frames': w['n'],
                      'states_per_frame': w['n_states'], 'form': 'FP64 NumPy restatement',
                      'l2': 'inputs larger than L2'},
           'cpu_baseline': {'value': v, 'unit': UNIT, 'cores': base['cores'], 'kind': 'port',
                            'sample': base['sample']},
           'e2e': {'value': v, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
           'reference_gpu': None if args.no_ref_gpu else reference_gpu(args, w, data, model)}
    print(json.dumps(out))
    return 0


def reference_gpu(args, w, data, model):
    """The reference's own kernels.cu on this GPU (built from the reference
    sources into oracle/_ref/), replaying emc.py's E-step loop and maxLP.py's
    per-pixel pattern search on a bounded sample; None-free dict with
    ``unavailable`` when the GPU or the built kernels are missing."""
    try:
        import torch
        if not torch.cuda.is_available():
            return {'unavailable': 'no CUDA device'}
        from oracle import emc_oracle as E
        from oracle.ref_gpu import replay
        from rspi import geometry
        if w['n_modes'] != 1 or w['cfg'].get('dense'):
            return {'unavailable': 'the reference runs one model on sparse photons only'}
        lib = replay.load()
        dev = torch.device('cuda', 0)
        size = w['size']
        ds = E.parse_photons(data['ones'], data['multi'], data['place_ones'], data['place_multi'],
                             data['count_multi'], size * size, True)
        _, pm = geometry.emc_masks(size)
        rd = replay.RefData(ds['ones'], ds['multi'], ds['place_ones'], ds['place_multi'],
                            ds['count_multi'], size, ds['bg'], E.get_scales(ds, True), pm, dev)
        r = w['recon']
        sx, sy, dia, _ = geometry.state_grid(geometry.parse_triple(r['shiftx']),
                                            geometry.parse_triple(r['shifty']),
                                            geometry.parse_triple(r['sphere_dia']))
        res = replay.time_iteration(lib, rd, torch.from_numpy(model).to(dev), sx, sy, dia,
                                    r['num_rot'])
        res['value'] = w['n'] * w['n_states'] / res['s_per_iteration']
        res['unit'] = UNIT
        return res
    except Exception as exc:   # reported, never fatal for the reference arm
        return {'unavailable': '%s: %s' % (type(exc).__name__, exc)}


def parity_block(rec, es, w, model0, dev, EStep):
    """One EMC iteration of the chosen (screened) form and of the plain FP64
    form from the same start model, compared over the whole likelihood
    matrix (every row x frame), the argmax, the per-frame maximum and
    log-sum-exp, and the model after the M-step (emc.py:134-157).  Returns
    the errors relative to FP64, or the reason the comparison was skipped."""
    import torch
    free, _ = torch.cuda.mem_get_info(dev)
    need = es.n_rows * w['n'] * 8 + es.chunk_rows * es.p_row * 8 + (1 << 30)
    if need > 0.9 * free:
        return {'skipped': 'the FP64 likelihood matrix (%.1f GB) does not fit beside the '
                           'chosen form\'s' % (es.n_rows * w['n'] * 8 / 1e9)}
    m_c = torch.from_numpy(model0).to(dev)
    es.run(m_c)
    maxll, rmax, logz = es.reduce()
    rec.phaser.run_from_rmax(m_c, rmax, w['num_rot'], rec.state_vals, rec.phaser_rot)
    screen0 = rec.phaser.mstep.screen
    rec.phaser.mstep.screen = False
    pe = EStep(rec.dset.photons, w['size'], w['num_rot'], rec.shiftx, rec.shifty,
               rec.sphere_dia, rec.probmask, rec.dset.bg.cpu().numpy(), n_modes=w['n_modes'],
               form='fp64', kernel='dynamic')
    m_p = torch.from_numpy(model0).to(dev)
    pe.run(m_p)
    maxll64, rmax64, logz64 = pe.reduce()
    rec.phaser.run_from_rmax(m_p, rmax64, w['num_rot'], rec.state_vals, rec.phaser_rot)
    rec.phaser.mstep.screen = screen0
    torch.cuda.synchronize()
    rec.dset.photons.err.check('parity iteration')
    # every entry of the FP32 matrix against FP64, in row chunks
    worst, nan_mismatch = 0., 0
    step = max(1, (1 << 28) // max(1, w['n']))
    cof = None if es.col_of_frame is None else es.col_of_frame.long()
    for r0 in range(0, es.n_rows, step):
        a = es.prob[r0:r0 + step]
        a = (a if cof is None else a.index_select(1, cof)).double()
        b = pe.prob[r0:r0 + step]
        nan_mismatch += int((a.isnan() != b.isnan()).sum().item())
        ok = ~b.isnan()
        if bool(ok.any()):
            worst = max(worst, float(((a - b).abs()[ok] / b.abs()[ok]).max().item()))

    def rel(x, y):
        return float(((x - y).abs() / y.abs().clamp_min(1e-300)).max().item())
    out = {'entries': es.n_rows * w['n'], 'll_rel_err_max': worst,
           'nan_mismatches': nan_mismatch,
           'argmax_identical': bool(torch.equal(rmax, rmax64)),
           'maxll_rel_err': rel(maxll, maxll64), 'logz_rel_err': rel(logz, logz64),
           'model_rel_err': rel(m_c, m_p),
           'candidates_rescored': getattr(es, 'n_candidates', None),
           'note': 'one iteration of each form from the start model; FP32 screened '
                   'likelihoods and FP64-rescored argmax/max/log-sum-exp vs the FP64 form, '
                   'model after the M-step vs the FP64 pattern search'}
    del pe
    torch.cuda.empty_cache()
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    from rspi import lib as rlib

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    w = workload(args.config, args.frames)
    t0 = time.time()
    data = generate_data(args.config, w, device=dev, rank=rank)
    t_gen = time.time() - t0
    tmp = tempfile.mkdtemp(prefix='rspi_bench_')
    # several ranks: each its own frames (photons_{rank}.npz), one job split
    # by frames (rspi/shard.py)
    cfgfile = write_inputs(tmp, w, data, args.form, args.slice_gb, args.screen_delta,
                           args.kernel if args.form != 'dense' else None, args.mstep,
                           not args.no_autotune and not args.warps,
                           rank=rank if world > 1 else None, slice_math=args.slice_math,
                           merge=args.merge, set_order=args.set_order)
    from emc import EMC
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        rec = EMC(cfgfile, device=dev)
    if args.warps:
        rec.estep.configure(warps=args.warps)
    if args.no_phaser_screen:
        rec.phaser.mstep.screen = False
    model0 = start_model(args.config, w)
    stream = torch.cuda.current_stream()

    es = rec.estep
    rec._dmodel.copy_(torch.from_numpy(model0).to(dev))
    l0 = rlib.launch_count
    rec._device_step()                      # one eager iteration: counts our launches
    torch.cuda.synchronize()
    kernels_per_step = rlib.launch_count - l0
    rec.device_step()                       # eager once more, then capture the graph
    for _ in range(max(0, args.warmup - 2)):
        rec.device_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    if not args.no_clocks:
        clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        rec.device_step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = kernels_per_step * args.steps
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    # the likelihood kernel alone: CUDA events on the launching stream around
    # each of its launches in one more E-step pass over the same buffers
    es.ll_events = []
    es.run(rec._dmodel)
    torch.cuda.synchronize()
    ll_ms = sum(a.elapsed_time(b) for a, b, _ in es.ll_events)
    ll_launches = len(es.ll_events)
    es.ll_events = None
    merge_info = None
    if rec.merger is not None:
        # the merge alone (row a10): CUDA events around one more merge of the
        # same E-step's posteriors
        es.reduce()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        rec.merger.run()
        m1.record(stream)
        torch.cuda.synchronize()
        n_pairs = int(es.cand_off[rec.dset.num_data].item()) if es.form != 'fp64' else None
        merge_info = {'ms': m0.elapsed_time(m1), 'posterior_pairs': n_pairs,
                      'p_min': rec.merger.p_min,
                      'note': 'posterior-weighted intensities of every (shift, diameter) '
                              'state, included in ms_per_step'}
    rec.dset.photons.err.check('bench')
    if world > 1:
        ms = max_over_ranks(ms, dev)
        dist.barrier()

    n_cand = getattr(rec.estep, 'n_candidates', None)
    ps = rec.phaser.mstep.stats.cpu().tolist()
    phaser_form = {'screen': rec.phaser.mstep.screen, 'iterations_screened': ps[0],
                   'iterations_fp64': ps[1], 'finalists': ps[2]}
    mem_gb = torch.cuda.max_memory_allocated(dev) / 1e9

    # e2e through the public API: host model in, host model + argmax out
    e2e = None
    if not args.no_e2e:
        # the same iterations as the device-timed loop: from the start model,
        # W untimed iterations, then K timed (the M-step's pattern search
        # depends on the model, so each iteration's work differs)
        rec.model = model0.copy().reshape(rec._model_shape())
        for _ in range(args.warmup):
            rec.run_iteration(None)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t_e0 = time.perf_counter()
        for _ in range(args.steps):
            rec.run_iteration(None)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t_e0) / args.steps
        if world > 1:
            e2e_s = max_over_ranks(e2e_s, dev)
        p = w['size'] ** 2 * w['n_modes']
        e2e = {'value': world * w['n'] * w['n_states'] / e2e_s, 'unit': UNIT,
               's_per_iteration': e2e_s, 'h2d_bytes_per_step': 16 * p,
               'd2h_bytes_per_step': 16 * p + 4 * w['n'],
               'api': 'EMC.run_iteration (model host->device, model + argmax device->host)'}

    # the plain form on the same data (FP64 slices and likelihoods,
    # warp-per-frame kernel, FP64 pattern search): first one iteration of each
    # form from the start model, compared entry by entry (the parity block),
    # then the plain form timed eagerly step by step
    plain, parity = None, None
    if world == 1 and not args.no_plain:
        from rspi.device import EStep
        rec._graph = None
        pe = None
        if es.form == 'screen':
            parity = parity_block(rec, es, w, model0, dev, EStep)
        # the chosen form's likelihood matrix, slices, candidates and graph
        # pool are released first: the matrices need not fit at once
        for name in ('prob', 'lsl', 'cand_d', 'cand_r', 'cand_ll', 'row_cand'):
            setattr(es, name, None)
        torch.cuda.empty_cache()

        def time_form(**kw):
            pe = EStep(rec.dset.photons, w['size'], w['num_rot'], rec.shiftx, rec.shifty,
                       rec.sphere_dia, rec.probmask, rec.dset.bg.cpu().numpy(),
                       n_modes=w['n_modes'], **kw)
            pmodel = torch.from_numpy(model0).to(dev)

            def pstep():
                pe.run(pmodel)
                pe.reduce()
                rec.phaser.run_from_rmax(pmodel, pe.rmax, w['num_rot'], rec.state_vals,
                                         rec.phaser_rot)
            for _ in range(min(args.warmup, 1)):
                pstep()
            torch.cuda.synchronize()
            p0 = torch.cuda.Event(enable_timing=True)
            p1 = torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            for _ in range(args.steps):
                pstep()
            p1.record(stream)
            torch.cuda.synchronize()
            pms = p0.elapsed_time(p1) / args.steps
            cands = getattr(pe, 'n_candidates', None)
            del pe
            torch.cuda.empty_cache()
            return pms, cands

        # the plain form searches every pattern candidate in FP64 as well
        screen0 = rec.phaser.mstep.screen
        rec.phaser.mstep.screen = False
        try:
            pms, _ = time_form(form='fp64', kernel='dynamic')
        except ValueError as e:
            # the plain form stages whole FP64 slice rows in shared memory
            # (at most ~28,900 likelihood pixels)
            pms = None
            plain = {'skipped': str(e)}
        rec.phaser.mstep.screen = screen0
        if pms is not None:
            plain = {'form': 'fp64 slices + FP64 likelihood matrix, warp-per-frame kernel, '
                             'FP64 pattern search',
                     'ms_per_step': pms, 'value': w['n'] * w['n_states'] / (pms * 1e-3),
                     'speedup_of_chosen': pms / ms}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0

    pk = peaks()
    sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
    roof, roof_gather, rows_per_launch = roofline_blocks(args, w, es, ll_ms, ll_launches, ms, clk,
                                                         pk, sm_count)
    esz = {0: 4, 1: 8, 2: 4}[es.slice_code]
    osz = 4 if es.prob_code == 0 else 8
    value = world * w['n'] * w['n_states'] / (ms * 1e-3)
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cb = cpu_baseline(w, {k: (v.cpu().numpy() if hasattr(v, 'cpu') else v) for k, v in data.items()},
                          model0[:w['size'] ** 2], args.cpu_seconds)
        cpu = {'value': w['n'] * w['n_states'] / cb['s_per_iteration'], 'unit': UNIT,
               'cores': cb['cores'], 'kind': 'port', 'sample': cb['sample'],
               's_per_iteration': cb['s_per_iteration']}
    out = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': ms, 's_per_iteration': ms / 1e3,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': {'fp64': 'f64', 'screen': 'f32 screen + f64 rescore',
                  'dense': ('u8 x fixed-point int8 GEMM (exact int32 accumulate)'
                            if es.form == 'dense' and es.dense_gemm == 'i8' else
                            'bf16 GEMM (f32 accumulate)') +
                           (' + f64 rescore' if getattr(es, 'rescore', True) else '')}[args.form],
        'data': 'synthetic (seeded generator with the configuration\'s shapes)',
        'config': {'workload': workload_name(args.config, w),
                   'frames': w['n'], 'states_per_frame': w['n_states'],
                   'form': args.form,
                   'parallelism': ('frame shards: %d ranks x %d frames, histogram all-reduce '
                                   'and pixel-split pattern search' % (world, w['n'])
                                   if world > 1 else 'single'),
                   'l2': 'inputs larger than L2 (slices %.1f GB, likelihoods %.1f GB per step)' %
                   (es.n_rows * es.p_row * esz / 1e9, es.n_rows * w['n'] * osz / 1e9)},
        'gpu_launches': launches,
        'cuda_graph': rec.use_graph,
        'roofline': roof,
        'roofline_gather': roof_gather,
        'clocks': clk,
        'e2e': e2e,
        'plain': plain,
        'parity': parity,
        'merge': merge_info,
        'tiling': {'warps_per_cta': getattr(es, 'warps', None),
                   'column_parts': es.parts() if es.form != 'dense' else None,
                   'rows_per_tile': getattr(es, 'tile', None),
                   'autotuned': bool(getattr(rec, 'tuning', None)),
                   'tuned_ms_per_row': (rec.tuning[1] if getattr(rec, 'tuning', None)
                                        else None)},
        'form': {'likelihood': args.form, 'kernel': es.kernel,
                 'set_order': getattr(es, 'set_order', None) if es.kernel == 'sets' else None,
                 'candidates_rescored': n_cand, 'rescore_window_nats': getattr(es, 'delta', None),
                 'pattern_search': phaser_form},
        'cpu_baseline': cpu,
        'setup_s': {'generate': t_gen},
        'device_memory_gb': mem_gb,
    }
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_adjoint_eval(args):
    """Config 3: config-2 data; the MaxLP NLL and its hand-written adjoint.
    Times NLL + gradient evaluations (FP32 terms, FP64 sums) and compares the
    L-BFGS update with the 64 x 32 polar grid search (and the reference's
    pattern search) on the final NLL and the FRC to the true object, from a
    start model 30% off the truth, with frame states from an E-step on it."""
    import torch
    from rspi import geometry, synth
    from rspi.adjoint import NLLProblem
    from rspi.device import DevicePhotons, EStep
    from rspi.evaluate import compare_updates
    dev = torch.device('cuda', 0)
    torch.cuda.set_device(dev)
    w = workload(2, args.frames)
    data = generate_data(2, w, device=dev)
    size, n, r = w['size'], w['n'], w['recon']
    ph = DevicePhotons(data['ones'], data['multi'], data['place_ones'], data['place_multi'],
                       data['count_multi'], size * size, True, dev)
    truth = data['fsample'] / float(data['rel_scale'])
    rng = np.random.default_rng(20260103)
    start = truth * (1 + 0.3 * rng.standard_normal(truth.size)) + 0.3 * np.abs(truth).mean() * (
        rng.standard_normal(truth.size) + 1j * rng.standard_normal(truth.size))
    sx, sy, dia, nst = geometry.state_grid(geometry.parse_triple(r['shiftx']),
                                          geometry.parse_triple(r['shifty']),
                                          geometry.parse_triple(r['sphere_dia']))
    _, pm = geometry.emc_masks(size)
    es = EStep(ph, size, r['num_rot'], sx, sy, dia, pm, np.zeros(size * size), form='screen')
    es.run(torch.from_numpy(start).to(dev))
    _, rmax, _ = es.reduce()
    sv = torch.from_numpy(geometry.state_values(sx, sy, dia, nst)).to(dev)
    del es
    torch.cuda.empty_cache()
    # throughput of one NLL + gradient evaluation (FP32 terms)
    fst = (rmax // r['num_rot']).long()
    vals = sv[fst]
    ang = ((rmax % r['num_rot']).double() * np.pi / r['num_rot']).cpu().numpy()
    prob = NLLProblem(ph, size, ang, precision='fp32')
    fre, fim = prob.model_pixels(start)
    args_t = (fre, fim, vals[:, 2].contiguous(), vals[:, 0].contiguous(),
              vals[:, 1].contiguous(), ph.scales)
    for _ in range(max(3, args.warmup)):
        prob.evaluate(*args_t, grad=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        prob.evaluate(*args_t, grad=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    t0 = time.perf_counter()
    cmp = compare_updates(ph, size, start, truth, rmax, r['num_rot'], sv, lbfgs_steps=50)
    t_cmp = time.perf_counter() - t0
    units = n * prob.n_pix
    out = {'metric': 'NLL + adjoint gradient evaluations/s (frame x pixel terms); final NLL and '
                     'FRC to truth: L-BFGS vs 64x32 polar grid', 'config': 3,
           'value': units / (ms * 1e-3), 'unit': 'frame*pixel/s', 'ms_per_step': ms,
           'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True,
           'dtype': 'f32 terms, f64 sums', 'data': 'synthetic, config-2 shapes',
           'workload': {'frames': n, 'pixels': prob.n_pix, 'size': size},
           'nll': cmp['nll'], 'frc_mean': cmp['frc_mean'], 'rescale': cmp['rescale'],
           'compare_s': t_cmp}
    print(json.dumps(out))
    return 0


def main():
    args = parse_args()
    if args.config == 3:
        return run_adjoint_eval(args)
    if args.impl == 'reference':
        return run_reference(args)
    return run_ours(args)


if __name__ == '__main__':
    sys.exit(main())
