#!/usr/bin/env python
"""In-plane rotation EMC with MaxLP on one B200 -- drop-in for ``recon.py``.

Same command line as the reference (recon.py:16-25):

    recon.py num_iter [-c config_file] [-d devices_file] [-s streams]

and the same outputs: ``output_folder/EMC.log`` with ``Iter time(s) change``
per iteration (recon.py:44-58), ``output_%03d`` per iteration and
``model_000.npy``, and the mean s/iteration excluding the first
(recon.py:61-65).  One process runs on one GPU; a devices file selects it
(first line), since the reference's MPI rank split is not used.
"""
import argparse
import os.path as op
import sys
import time

import numpy as np
import torch

sys.path.insert(0, op.dirname(op.abspath(__file__)))
from emc import EMC  # noqa: E402


def main(argv=None):
    '''Command-line entry point: read the options, build the EMC reconstructor and run it'''
    parser = argparse.ArgumentParser(description='In-plane rotation EMC')
    parser.add_argument('num_iter', type=int, help='Number of iterations')
    parser.add_argument('-c', '--config_file', default='emc_config.ini',
                        help='Path to configuration file (default: emc_config.ini)')
    parser.add_argument('-d', '--devices', help='Path to devices file')
    parser.add_argument('-s', '--streams', type=int, default=4,
                        help='Number of streams to use (default=4)')
    args = parser.parse_args(argv)

    if args.devices is None:
        print('Running on default device 0')
        dev = 0
    else:
        with open(args.devices) as f:
            dev = int(f.readlines()[0].strip())
        print('Rank 0: (Device %d)' % dev)
    torch.cuda.set_device(dev)
    sys.stdout.flush()

    recon = EMC(args.config_file, num_streams=args.streams)
    logf = open(op.join(recon.output_folder, 'EMC.log'), 'w')
    logf.write('Iter  time(s)  change\n')
    logf.flush()
    avgtime = 0.
    numavg = 0
    for i in range(args.num_iter):
        m0 = np.array(recon.model, copy=True)
        stime = time.time()
        recon.run_iteration(i + 1)
        etime = time.time()
        sys.stderr.write('\r%d/%d (%f s)\n' % (i + 1, args.num_iter, etime - stime))
        norm = float(np.linalg.norm(np.asarray(recon.model) - m0))
        logf.write('%-6d%-.2e %e\n' % (i + 1, etime - stime, norm))
        print('Change from last iteration: ', norm)
        logf.flush()
        if i > 0:
            avgtime += etime - stime
            numavg += 1
    if numavg > 0:
        print('\n%.4e s/iteration on average' % (avgtime / numavg))
    logf.close()
    return recon


if __name__ == '__main__':
    main()
