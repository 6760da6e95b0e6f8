"""Stand-in for cupyx (SciPy-backed)."""
