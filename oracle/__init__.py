"""FP64 NumPy oracle for the RefSPI-MaxLP reconstruction hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
package.  It is used by ``tests/``, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` -- always as the
checker (or the timed CPU stand-in for the reference), never as the thing that
produces a product result.

Every function restates the reference equations in FP64 and cites the
reference file:line it follows (paths are relative to the RefSPI-MaxLP
project root).  Pinning: the restatement is checked against golden vectors
produced by running the reference's own Python code (``emc.py``, ``maxLP.py``,
``dset.py``) with NumPy standing in for CuPy and with the reference's own
``kernels.cu`` compiled for the CPU (``oracle/ref_cpu``); see
``tests/golden/make_golden.py``.

Modules
-------
emc_oracle    E-step: photon parsing, states, masks, holographic slices,
              rotated log-slices, log-likelihood, argmax/unravel, posterior,
              merge (a1-a10).
maxlp_oracle  M-step: per-pixel photons, reference form factor, rescale,
              per-candidate log-likelihood, pattern search, phaser (a11-a14).
adjoint_oracle  FP64 negative log-likelihood used for gradient checks (a16).
"""
