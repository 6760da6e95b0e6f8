#!/usr/bin/env python
"""EMC reconstructor on one B200 -- drop-in for the reference ``emc.py``.

``EMC(config_file, num_streams=4)`` reads the same ``[emc]`` keys
(emc.py:57-80), builds the same state grid and masks (emc.py:67-98) and keeps
the reference's attributes and methods: ``run_iteration(iternum=None)``,
``_calculate_prob``, ``_get_rmax``, ``_unravel_rmax``, ``save_output``,
``_random_model``, ``ramp``, ``sphere``; ``model`` is a host complex128
array and ``rmax`` a host int32 array, as in the reference.  The E-step and
the MaxLP M-step run in librspi on the GPU; ``prob`` is a torch CUDA tensor
(rows ``s*num_rot + j``, columns frames).

Optional ``[emc]`` keys beyond the reference: ``form`` (``fp64``: FP64
slices and FP64 likelihood matrix; ``screen``, the default: FP32 screening pass with
FP64 rescoring of every state that can be the argmax (and, with
``screen_delta`` > 0, carry posterior mass), same argmax/maximum as
``fp64``; ``dense``: frames stored
densely, likelihood as a tensor-core GEMM, ``dense_gemm`` = ``auto`` /
``i8`` (exact fixed point) / ``bf16`` (hi + lo split), ``dense_rescore``
(default true: FP64 rescoring of the candidates as in ``screen``)),
``kernel`` (the likelihood kernel: ``sets`` (the screened form's
default: one lane per frame, 32 frames per warp), ``quad4`` (four frames
per warp) or ``stream`` for the screened form, ``stream`` (default) or
``dynamic`` for ``fp64``), ``slice_math`` (``fp32``, the
frame-set kernel's default: its log-slices interpolated and logged in FP32
within a bound the candidate threshold covers; ``fp64``: computed in FP64,
stored in FP32, the other kernels' only choice), ``set_order``
(``grouped``, the default: each quarter warp's eight frames picked among
256 of alike photon count so that their bank-class totals stay close to
their mean; ``rank``: taken in rank order),
``merge`` (default false: true adds each iteration's posterior-weighted
intensities of every (shift, diameter) state, the reference's unused
``merge_all`` / ``slice_merge`` kernels (kernels.cu:84-152), to
output_%03d.h5 as ``intens``; ``screen_delta`` then defaults to 20),
``screen_delta``
(default 0: FP64 rescoring of the states that can be the argmax, which is
what the hard-argmax iteration uses; 20: also every state within 20 nats of
it, so that ``logz`` equals the FP64 form's -- the posterior consumers'
setting), ``states_per_tile``, ``warps_per_cta``, ``phaser_iter``
(default 10, maxLP.py:320,335), ``phaser_screen`` (default true: FP32
screening of the pattern-search candidates, FP64 for the finalists, same
chosen candidates as false), ``slice_budget_gb`` (rotated slices are built
in chunks of at most this size, default 8), ``cuda_graph`` (capture the whole
device iteration once and replay it, default true), ``autotune`` (pick the
likelihood kernel's tiling by timing it on the first iteration's slices,
cached per geometry, default true), ``mstep``
(``pattern``, the default: the MaxLP pattern search; ``grid``: the polar grid
search of the pixel NLL; ``lbfgs``: L-BFGS on that NLL through its
hand-written adjoint, ``lbfgs_steps`` iterations, default 50;
``grid+lbfgs``: the grid, then L-BFGS).

``num_modes`` (emc.py:59, parsed but unused by the reference) reconstructs
that many models at once: the (shift, diameter) grid is repeated per mode,
likelihood rows are ``(m*S0 + s)*num_rot + j``, each frame's argmax picks a
mode as well as a state, and MaxLP updates each mode from the frames that
chose it.  ``model`` is then a (num_modes, size**2) array and
``output_%03d.h5`` holds ``model`` as (num_modes, size, size) plus each
frame's mode in ``modes``.

Several GPUs: run one process per GPU inside an initialised
torch.distributed group (NCCL).  The reference splits states over MPI ranks
(emc.py:143,171,207-216); here each rank takes a contiguous block of the
frames (or its own file when ``in_photons_file`` contains ``{rank}``),
computes every state for them with no exchange, and the M-step sums the
pixel histograms over ranks and splits the pattern search by pixels
(rspi/shard.py): model and argmax are those of one GPU, bit for bit.  Rank
0 writes the output files; ``prob`` holds the rank's own frames.
"""
import configparser
import os.path as op
import sys
import time

import numpy as np
import torch

sys.path.insert(0, op.dirname(op.abspath(__file__)))
from dset import Dataset  # noqa: E402
from maxLP import MaxLPhaser  # noqa: E402
from rspi import geometry  # noqa: E402
from rspi import h5lite  # noqa: E402
from rspi import shard  # noqa: E402
from rspi.device import cur_stream, ptr  # noqa: E402
from rspi.lib import call  # noqa: E402
from rspi.device import EStep  # noqa: E402

P_MIN = 1.e-6   # emc.py:20
RSPI_ERR_CAPACITY = -5   # include/rspi.h


class EMC():
    '''Reconstructor object using parameters from config file

    Args:
        config_file (str): Path to configuration file
        num_streams (int): accepted for compatibility; all work is issued on
            torch's current CUDA stream
    '''
    def __init__(self, config_file, num_streams=4, device=None):
        self.num_streams = num_streams
        # several ranks of an initialised torch.distributed group split the
        # frames (rspi/shard.py); one rank is the reference's one-process run
        self.rank, self.num_proc = shard.world()
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.mem_size = torch.cuda.get_device_properties(self.device).total_memory

        config = configparser.ConfigParser()
        config.read(config_file)
        self._parse_params(config, op.dirname(config_file))
        self._generate_states(config)
        self._generate_masks()

        self._parse_data()
        self.phaser = MaxLPhaser(self.photons_file, size=self.size, dataset=self.dset,
                                 num_iter=self.phaser_iter, num_modes=self.num_modes,
                                 screen=self.phaser_screen)
        if self.num_proc > 1:
            if self.mstep_kind != 'pattern':
                raise ValueError('emc:mstep %s runs on one GPU' % self.mstep_kind)
            self.phaser.mstep.shard = shard.ShardedMStep(self.phaser.mstep)
        self._init_model()

        self.estep = EStep(self.dset.photons, self.size, self.num_rot, self.shiftx,
                           self.shifty, self.sphere_dia, self.probmask,
                           self.dset.bg.cpu().numpy(), form=self.form,
                           states_per_tile=self.states_per_tile, warps=self.warps_per_cta,
                           delta=self.screen_delta,
                           slice_budget_bytes=int(self.slice_budget_gb * (1 << 30)),
                           n_modes=self.num_modes, dense_gemm=self.dense_gemm,
                           dense_rescore=self.dense_rescore, kernel=self.kernel,
                           slice_math=self.slice_math, set_order=self.set_order)
        self.merger = None
        self.intens = None
        if self.merge_intens:
            if self.num_proc > 1:
                raise ValueError('emc:merge runs on one GPU')
            from rspi.device import Merge
            self.merger = Merge(self.estep, p_min=P_MIN)
        self.state_vals = torch.from_numpy(self._state_values).to(self.device)
        self.phaser_rot = torch.from_numpy(geometry.phaser_rotation_table(
            np.arange(self.num_rot) * np.pi / self.num_rot)).to(self.device)
        self.rmax = None
        self._tuned = not self.autotune or self.form == 'dense'
        npix = self.size ** 2 * self.num_modes
        self._dmodel = torch.empty(npix, dtype=torch.complex128, device=self.device)
        self._host_model = torch.empty(npix, dtype=torch.complex128, pin_memory=True)
        self._host_rmax = torch.empty(self.dset.num_data, dtype=torch.int32, pin_memory=True)
        self._graph = None

    def _parse_params(self, config, start_dir):
        '''emc.py:57-65, plus the optional precision/tiling keys'''
        self.size = config.getint('emc', 'size')
        self.num_modes = config.getint('emc', 'num_modes', fallback=1)
        if self.num_modes < 1:
            raise ValueError('emc:num_modes must be at least 1')
        self.num_rot = config.getint('emc', 'num_rot')
        self.photons_file = op.join(start_dir, config.get('emc', 'in_photons_file'))
        self.output_folder = op.join(start_dir, config.get('emc', 'output_folder'))
        self.log_file = op.join(start_dir, config.get('emc', 'log_file'))
        self.need_scaling = config.getboolean('emc', 'need_scaling', fallback=False)
        self.form = config.get('emc', 'form', fallback='screen')
        if self.form not in ('fp64', 'screen', 'dense'):
            raise ValueError('emc:form must be fp64, screen or dense')
        # merge: the posterior-weighted intensities of every (shift, diameter)
        # state (a10), written as output_%03d.h5's ``intens``; the posteriors
        # above P_MIN need FP64 values within 13.8 nats of each maximum, so the
        # rescoring window defaults to 20 nats then
        self.merge_intens = config.getboolean('emc', 'merge', fallback=False)
        self.screen_delta = config.getfloat('emc', 'screen_delta',
                                            fallback=20. if self.merge_intens else 0.)
        self.states_per_tile = config.getint('emc', 'states_per_tile', fallback=0) or None
        self.warps_per_cta = config.getint('emc', 'warps_per_cta', fallback=32)
        self.phaser_iter = config.getint('emc', 'phaser_iter', fallback=10)
        self.phaser_screen = config.getboolean('emc', 'phaser_screen', fallback=True)
        self.slice_budget_gb = config.getfloat('emc', 'slice_budget_gb', fallback=8.)
        self.use_graph = config.getboolean('emc', 'cuda_graph', fallback=True)
        self.dense_gemm = config.get('emc', 'dense_gemm', fallback='auto')
        self.dense_rescore = config.getboolean('emc', 'dense_rescore', fallback=True)
        self.autotune = config.getboolean('emc', 'autotune', fallback=True)
        self.kernel = config.get('emc', 'kernel', fallback=None) or None
        self.slice_math = config.get('emc', 'slice_math', fallback='').strip() or None
        self.set_order = config.get('emc', 'set_order', fallback='grouped').strip()
        self.mstep_kind = config.get('emc', 'mstep', fallback='pattern')
        if self.mstep_kind not in ('pattern', 'grid', 'lbfgs', 'grid+lbfgs'):
            raise ValueError('emc:mstep must be pattern, grid, lbfgs or grid+lbfgs')
        if self.mstep_kind != 'pattern' and self.num_modes != 1:
            raise ValueError('emc:mstep %s takes one mode' % self.mstep_kind)
        self.lbfgs_steps = config.getint('emc', 'lbfgs_steps', fallback=50)

    def _generate_states(self, config):
        '''emc.py:67-87'''
        dia = geometry.parse_triple(config.get('emc', 'sphere_dia'))
        sx = geometry.parse_triple(config.get('emc', 'shiftx'))
        sy = geometry.parse_triple(config.get('emc', 'shifty'))
        self.shiftx, self.shifty, self.sphere_dia, self.num_states = geometry.state_grid(sx, sy, dia)
        print(self.num_states.prod(), 'sampled states')
        self.x_ind, self.y_ind, self.rad = geometry.detector_radius(self.size)
        self._state_values = geometry.state_values(self.shiftx, self.shifty, self.sphere_dia,
                                                   self.num_states)

    def _generate_masks(self):
        '''emc.py:89-98'''
        self.invmask, self.probmask = geometry.emc_masks(self.size)
        self.intinvmask = self.invmask.astype('i4')

    def _parse_data(self):
        '''emc.py:109-118'''
        stime = time.time()
        self.dset = Dataset(self.photons_file, self.size ** 2, self.need_scaling,
                            device=self.device, shard=self.num_proc > 1)
        self.powder = self.dset.get_powder()
        etime = time.time()
        print('%d frames with %.3f photons/frame (%.3f s) (%.2f MB)' %
              (self.dset.num_data, self.dset.mean_count, etime - stime, self.dset.mem / 1024 ** 2))
        sys.stdout.flush()

    def _init_model(self):
        '''emc.py:120-132'''
        self._random_model()
        np.save(op.join(self.output_folder, 'model_000.npy'), self.model)
        self.scales = self.dset.photons.scales

    def run_iteration(self, iternum=None):
        '''Run one iteration of EMC: likelihoods of every state, most likely
        state per frame, MaxLP M-step, output (emc.py:134-157).  The model goes
        to the device, the whole device iteration runs (replayed from a CUDA
        graph after the first iteration) and model and rmax come back.'''
        self._host_model.numpy()[:] = np.asarray(self.model, dtype=np.complex128).ravel()
        self._dmodel.copy_(self._host_model, non_blocking=True)
        self.device_step()
        self._host_rmax.copy_(self.estep.rmax, non_blocking=True)
        self._host_model.copy_(self._dmodel, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        err = self.dset.photons.err
        if self._graph is not None and int(err.t.item()) == RSPI_ERR_CAPACITY:
            # the candidate buffers sized by the eager iteration were too
            # small inside the graph: redo the iteration eagerly (which grows
            # them) and capture again next time; any other error is raised
            err.t.zero_()
            self._graph = None
            self._dmodel.copy_(torch.from_numpy(np.asarray(self.model, dtype=np.complex128).ravel()))
            self._device_step()
            if self.merger is not None:
                self.intens = self.merger.run()
            self._host_rmax.copy_(self.estep.rmax)
            self._host_model.copy_(self._dmodel)
        err.check('EMC iteration')
        if self.num_proc > 1:
            # every rank's argmax, in frame order (the model is the same on
            # every rank)
            self.rmax = shard.gather_frames(self.estep.rmax, self.dset.num_data_global).cpu() \
                .numpy().astype('i4')
        else:
            self.rmax = self._host_rmax.numpy().copy()
        self.model = self._host_model.numpy().copy().reshape(self._model_shape())
        if self.rank == 0:
            self.save_output(self.model, iternum, intens=self.intens)

    def _device_step(self):
        '''One iteration on device buffers: E-step, reduction, M-step.'''
        self._estep_part()
        self._mstep_part()

    def _estep_part(self):
        self.estep.run(self._dmodel)
        self.estep.reduce()

    def _mstep_part(self):
        '''The M-step on the E-step's argmax: the MaxLP pattern search
        (maxLP.py:304-340, ``mstep = pattern``), or after its ring pass and
        global rescale (maxLP.py:317-330) the polar grid search of the pixel
        NLL (``grid``), L-BFGS on that NLL through its hand-written adjoint
        (``lbfgs``, ``lbfgs_steps`` iterations), or the grid then L-BFGS
        (``grid+lbfgs``) over the main phaser pixels.'''
        if self.mstep_kind == 'pattern':
            self.phaser.run_from_rmax(self._dmodel, self.estep.rmax, self.num_rot,
                                      self.state_vals, self.phaser_rot)
            return
        from rspi.adjoint import NLLProblem, lbfgs_update
        ms = self.phaser.mstep
        n_ref = self.state_vals.shape[0]
        ms.frame_params_from_rmax(self.estep.rmax, self.num_rot, n_ref)
        ms.run(self._dmodel, self.state_vals, self.phaser_rot, main=False)
        scale = self.dset.photons.scales * ms.rescale[0]
        if 'grid' in self.mstep_kind:
            ms.grid(self._dmodel, self.state_vals, self.phaser_rot, scale)
        if 'lbfgs' in self.mstep_kind:
            vals = self.state_vals[ms.fstate.long()]
            ang = (ms.frot.double() * np.pi / self.num_rot).cpu().numpy()
            prob = NLLProblem(self.dset.photons, self.size, ang, precision='fp32')
            out, self.mstep_nll, _ = lbfgs_update(
                prob, self._dmodel.cpu().numpy(), vals[:, 2].cpu().numpy(),
                vals[:, 0].cpu().numpy(), vals[:, 1].cpu().numpy(), scale.cpu().numpy(),
                steps=self.lbfgs_steps)
            self._dmodel.copy_(torch.from_numpy(out))

    def device_step(self):
        '''The iteration on the device model buffer ``_dmodel``: eager the
        first time (which sizes every buffer and checks capacities), then
        captured once into a CUDA graph and replayed; with ``merge`` the
        posterior-weighted intensities of the iteration's E-step follow
        (eagerly: the merge sizes its pair buffers on the host).'''
        self._iteration()
        if self.merger is not None:
            self.intens = self.merger.run()

    def _iteration(self):
        if not self._tuned:
            # the likelihood kernel's tiling, timed on this model's slices
            from rspi import autotune
            self.estep.slices(self._dmodel)
            self.tuning = autotune.tune(self.estep)[:2]
            self._tuned = True
        if not self.use_graph:
            self._device_step()
            return
        # the graph holds the whole iteration, or the E-step only with an
        # adjoint-driven M-step (host-side L-BFGS line searches) or with
        # frames split over ranks (collectives in the M-step)
        whole = self.mstep_kind == 'pattern' and self.num_proc == 1
        part = self._device_step if whole else self._estep_part
        if self._graph is not None:
            self._graph.replay()
            if not whole:
                self._mstep_part()
            return
        self._device_step()
        torch.cuda.current_stream(self.device).synchronize()
        model_after = self._dmodel.clone()
        self.estep.check_capacity = False
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            with torch.cuda.graph(graph, stream=side):
                part()
        torch.cuda.current_stream(self.device).wait_stream(side)
        self.estep.check_capacity = True
        self._dmodel.copy_(model_after)   # capture does not execute: keep the eager result
        self._graph = graph

    def _calculate_prob(self, dmodel, views=None, drange=None):
        '''Likelihood of every frame in every state into ``prob``
        (emc.py:159-205 with calc_prob_all, kernels.cu:116-137)'''
        if drange is not None and tuple(drange) != (0, self.dset.num_data):
            raise ValueError('frame ranges are not supported: all frames are processed')
        self.estep.run(dmodel)
        return self.prob

    @property
    def prob(self):
        '''Likelihood of every frame (columns) in every state (rows
        ``s*num_rot + j``), emc.py's ``prob``; a device tensor in frame order
        (a reordered copy when the likelihood kernel keeps frames in set
        order)'''
        return self.estep.frame_prob()

    def _get_rmax(self):
        '''First-index argmax per frame (emc.py:207-216; one rank)'''
        maxll, rmax, logz = self.estep.reduce()
        self.max_exp = maxll
        self.logz = logz
        self.rmax = rmax.cpu().numpy().astype('i4')

    def _unravel_rmax(self, rmax):
        '''Grid values of the chosen states (emc.py:218-224); the mode of
        each frame is ``_rmax_modes(rmax)``'''
        rmax = np.asarray(rmax)
        s0 = (rmax // self.num_rot) % len(self._state_values)
        ang = rmax % self.num_rot
        vals = self._state_values[s0]
        return vals[:, 0], vals[:, 1], vals[:, 2], ang * np.pi / self.num_rot

    def _rmax_modes(self, rmax):
        '''Mode of each frame's most likely state'''
        return (np.asarray(rmax) // self.num_rot // len(self._state_values)).astype('i4')

    def _model_shape(self):
        npix = self.size ** 2
        return (npix,) if self.num_modes == 1 else (self.num_modes, npix)

    def save_output(self, model, iternum, intens=None):
        '''``model.npy``, or ``output_%03d.h5`` (HDF5, written by rspi.h5lite)
        with the datasets model, angles, diameters, shifts and optional
        intens (emc.py:226-239)'''
        if iternum is None:
            np.save(op.join(self.output_folder, 'model.npy'), self.model)
            return
        sx_vals, sy_vals, dia_vals, ang_vals = self._unravel_rmax(self.rmax)
        shape = (self.size,) * 2 if self.num_modes == 1 else (self.num_modes,) + (self.size,) * 2
        out = {'model': np.asarray(self.model).reshape(shape),
               'angles': ang_vals, 'diameters': dia_vals,
               'shifts': np.array([sx_vals, sy_vals]).T}
        if self.num_modes > 1:
            out['modes'] = self._rmax_modes(self.rmax)
        if intens is not None:
            out['intens'] = intens.cpu().numpy() if torch.is_tensor(intens) else np.asarray(intens)
        h5lite.write_datasets(op.join(self.output_folder, 'output_%.3d.h5' % iternum), out)

    def _random_model(self):
        '''emc.py:241-242 (one such model per mode; with several ranks rank
        0's, so that every rank starts from the same model)'''
        shape = self._model_shape()
        self.model = np.random.random(shape) + 1j * np.random.random(shape)
        if self.num_proc > 1:
            m = torch.from_numpy(np.ascontiguousarray(self.model).ravel()).to(self.device)
            torch.distributed.broadcast(torch.view_as_real(m), 0)
            self.model = m.cpu().numpy().reshape(shape)

    def ramp(self, n):
        '''Shift phase ramp of state n (emc.py:244-245), a complex128 CUDA
        tensor of P pixels'''
        out = torch.empty(self.size ** 2, dtype=torch.complex128, device=self.device)
        call('rspi_sphere_ramp', self.size, float(self.shiftx[n]), float(self.shifty[n]), 0.,
             None, ptr(out), cur_stream())
        return out

    def sphere(self, n, diameter=None):
        '''Sphere form factor of state n or of a diameter (emc.py:247-254), a
        float64 CUDA tensor of P pixels'''
        dia = diameter if n is None else self.sphere_dia[n]
        out = torch.empty(self.size ** 2, dtype=torch.float64, device=self.device)
        call('rspi_sphere_ramp', self.size, 0., 0., float(dia), ptr(out), None, cur_stream())
        return out
