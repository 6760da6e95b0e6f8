"""Stand-in for mpi4py with a single rank."""
