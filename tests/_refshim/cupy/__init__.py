"""NumPy-backed stand-in for the ``cupy`` module, used only to run the
reference KSig package on the CPU when generating golden fixtures.

KSig imports ``cupy as cp`` and calls array functions that share NumPy's
names and semantics; this module re-exports NumPy under that name and adds
the few CuPy-only entry points KSig touches (``asnumpy``, ``cuda.Device``
attributes, ``random.RandomState``).  It is test infrastructure: nothing in
the ``ksig_b200`` package imports it.
"""
import numpy as _np
from numpy import *  # noqa: F401,F403
from numpy import ndarray  # noqa: F401

from . import random  # noqa: F401
from . import cuda  # noqa: F401
from . import fft  # noqa: F401


def asnumpy(a, *args, **kwargs):
  return _np.asarray(a)


def asarray(a, *args, **kwargs):
  return _np.asarray(a, *args, **kwargs)


isscalar = _np.isscalar
