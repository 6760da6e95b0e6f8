"""Stand-in for cupyx.scipy."""
