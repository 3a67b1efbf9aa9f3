"""``cupy.fft`` stand-in."""
from numpy.fft import *  # noqa: F401,F403
