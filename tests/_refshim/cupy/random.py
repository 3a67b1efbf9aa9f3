"""``cupy.random`` stand-in: NumPy's legacy RandomState."""
from numpy.random import *  # noqa: F401,F403
from numpy.random import RandomState  # noqa: F401
