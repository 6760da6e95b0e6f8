"""Frame-sharded EMC over several GPUs: one process per GPU (torch.distributed,
NCCL over NVLink; any backend for the host logic).

The reference splits the *states* over MPI ranks and reduces every frame's
maximum and argmax with Allreduce(MAX) (emc.py:143,171,207-216), and runs
MaxLP redundantly.  Here the *frames* are split, which needs no exchange in
the E-step at all (each rank keeps every state for its frames):

* set-up: each rank holds its frames' photons; the dataset-wide statistics
  the reference computes over all frames -- the mean photon count behind
  the per-frame scales (emc.py:129-132, dset.py:46-48) and the powder
  (dset.py:74-83) -- come from one all-reduce of exact integer sums, so they
  are bit-identical to a single GPU's;
* E-step and argmax: local (rank-local likelihood columns);
* M-step: the photon histograms of the phaser pixels (per reference state)
  and the frame counts per state are sums over frames: one all-reduce (SUM)
  of integers, after which every rank holds the single-GPU histogram; the
  ring pass and the global rescale run on every rank (identical), the main
  pass is split by pixels and the updated pixels are combined with one
  all-reduce in which every other rank contributes exact zeros.

The models and argmaxes are therefore bit-identical to the single-GPU
iteration on the same frames.
"""
import numpy as np
import torch
import torch.distributed as dist

from .device import DevicePhotons, call, cur_stream, ptr

_f64 = torch.float64


def world():
    """(rank, world size) of the initialised process group, or (0, 1)."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def block_range(n, rank, size):
    """Contiguous block ``[lo, hi)`` of ``n`` items owned by ``rank`` of
    ``size`` (the first ``n % size`` ranks hold one more)."""
    n, rank, size = int(n), int(rank), int(size)
    if not (0 <= rank < size):
        raise ValueError('rank %d outside a world of %d' % (rank, size))
    return n * rank // size, n * (rank + 1) // size


def frames_of_host(host, lo, hi):
    """Frames ``[lo, hi)`` of a host photon dict (the ``read_photons``
    layout)."""
    ones = np.asarray(host['ones'])
    multi = np.asarray(host['multi'])
    o0, o1 = int(ones[:lo].sum()), int(ones[:hi].sum())
    m0, m1 = int(multi[:lo].sum()), int(multi[:hi].sum())
    out = dict(host)
    out.update(num_data=hi - lo, ones=ones[lo:hi], multi=multi[lo:hi],
               place_ones=np.asarray(host['place_ones'])[o0:o1],
               place_multi=np.asarray(host['place_multi'])[m0:m1],
               count_multi=np.asarray(host['count_multi'])[m0:m1])
    if host.get('frames') is not None:
        out['frames'] = host['frames'][lo:hi]
    return out


def _all_reduce(t, group=None):
    """SUM all-reduce of ``t`` in place (complex tensors as real pairs)."""
    if t.is_complex():
        dist.all_reduce(torch.view_as_real(t), group=group)
    else:
        dist.all_reduce(t, group=group)
    return t


def combine_stats(photons, n_frames, powder_sums, counts, need_scaling, group=None):
    """Dataset-wide statistics from this rank's exact integer sums: its
    photon total (ones + multi counts), frame count, per-pixel photon sums
    (float64 holding integers) and per-frame counts.  Returns (frames over
    all ranks, mean count, this rank's scales, powder) computed as a single
    GPU computes them: mean = total / N (dset.py:46-48), scale_d = count_d /
    mean (emc.py:129-132), powder = sums / N (dset.py:74-83)."""
    dev = powder_sums.device
    tot = torch.tensor([int(photons), int(n_frames)], dtype=torch.int64, device=dev)
    _all_reduce(tot, group)
    n_all, total = int(tot[1].item()), int(tot[0].item())
    mc = float(total) / float(n_all)
    scales = counts.to(_f64) / mc if need_scaling else torch.ones_like(counts, dtype=_f64)
    sums = powder_sums.clone()
    _all_reduce(sums, group)
    return n_all, mc, scales, sums / float(n_all)


def set_global_stats(ph, group=None):
    """Replace ``ph``'s frame-local mean count, scales and powder by the
    dataset-wide ones (``combine_stats`` of its exact sums)."""
    sums = torch.empty(ph.num_pix, dtype=_f64, device=ph.device)
    call('rspi_powder', ptr(ph.place_ones), ph.place_ones.numel(), ptr(ph.place_multi),
         ptr(ph.count_multi), ph.place_multi.numel(), ph.num_pix, 1, ptr(sums), ptr(ph.err.t),
         cur_stream())
    ph.err.check('sharded photon statistics')
    photons = int(ph.totals[0].item()) + int(ph.totals[2].item())
    n_all, mc, scales, powder = combine_stats(photons, ph.num_data, sums, ph.counts,
                                              ph.need_scaling, group)
    ph.num_data_global = n_all
    ph.mean_count = mc
    ph.mean_count_t.fill_(mc)
    ph.scales.copy_(scales)
    ph.powder.copy_(powder)
    return ph


def shard_photons(host, num_pix, need_scaling, device, group=None, pre_sharded=False):
    """This rank's frames on the device with dataset-wide statistics.
    ``host`` is the whole dataset (its frames split in contiguous blocks)
    or, with ``pre_sharded``, this rank's own frames."""
    rank, size = world()
    if not pre_sharded:
        lo, hi = block_range(host['num_data'], rank, size)
        host = frames_of_host(host, lo, hi)
    else:
        lo = None
    if host['num_data'] == 0:
        raise ValueError('rank %d holds no frames' % rank)
    ph = DevicePhotons(host['ones'], host['multi'], host['place_ones'], host['place_multi'],
                       host['count_multi'], num_pix, need_scaling, device,
                       frames=host.get('frames'))
    ph.frame_offset = lo
    return set_global_stats(ph, group)


class ShardedMStep:
    """Collectives of the M-step over frame shards, plugged into an MStep:
    the histogram and state counts are summed over ranks, the main pass runs
    on this rank's block of the main pixels and the updated pixels are
    gathered by an all-reduce of exact zeros elsewhere."""

    def __init__(self, mstep, group=None):
        self.ms = mstep
        self.group = group
        self.rank, self.size = world()

    def reduce_histogram(self, hist, nstate):
        _all_reduce(hist, self.group)
        _all_reduce(nstate, self.group)

    def main_block(self):
        return block_range(self.ms.n_main, self.rank, self.size)

    def gather_main(self, fconv, pixels):
        """Pixels ``pixels`` (this rank's block of the main pass) of every
        model to all ranks."""
        npix = self.ms.size ** 2
        f = fconv.view(-1, npix)
        buf = torch.zeros_like(f)
        buf[:, pixels.long()] = f[:, pixels.long()]
        _all_reduce(buf, self.group)
        allmain = self.ms.main.long()
        f[:, allmain] = buf[:, allmain]
        return fconv


def gather_frames(x, n_total, group=None):
    """Per-frame values of every rank's contiguous block, in frame order
    (all ranks receive the whole array, on ``x``'s device)."""
    rank, size = world()
    dev = x.device
    if dev.type == 'cuda' and dist.get_backend(group) == 'gloo':
        return gather_frames(x.cpu(), n_total, group).to(dev)   # gloo gathers host tensors
    counts = torch.tensor([x.numel()], dtype=torch.int64, device=x.device)
    sizes = [torch.zeros_like(counts) for _ in range(size)]
    dist.all_gather(sizes, counts, group=group)
    sizes = [int(s.item()) for s in sizes]
    if sum(sizes) != n_total:
        raise ValueError('frame blocks hold %d frames, expected %d' % (sum(sizes), n_total))
    m = max(sizes)
    pad = torch.zeros(m, dtype=x.dtype, device=x.device)
    pad[:x.numel()] = x
    parts = [torch.zeros_like(pad) for _ in range(size)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)])
