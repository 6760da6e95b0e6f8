"""Stand-in for cupyx.scipy.ndimage."""
from scipy.ndimage import *  # noqa: F401,F403
