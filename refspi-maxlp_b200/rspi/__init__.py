"""Internals of the B200 RefSPI-MaxLP hot path.

lib         ctypes binding of librspi.so (include/rspi.h)
device      device-resident photons and the E-step / M-step pipelines
geometry    static grids, masks and angle tables (host, set-up only)
photonfile  photons-file container with the reference's dataset names
synth       seeded synthetic data with the benchmark configurations
"""
