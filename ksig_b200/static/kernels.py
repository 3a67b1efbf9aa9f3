"""Static (state-space) kernels used inside the signature kernels.

Mirrors ``ksig.static.kernels`` (ksig/static/kernels.py).  Inside
``SignatureKernel`` / ``SignaturePDEKernel`` a static kernel is never
materialised: its parameters select the epilogue of the fused CUDA Gram
(``kind`` and ``param`` below).  Calling a static kernel directly evaluates
its Gram on the device with PyTorch tensor ops, as a convenience outside the
signature-kernel path.
"""

from abc import ABCMeta

import numpy as np
import torch

from .. import utils
from .._lib import STATIC_LINEAR, STATIC_RBF


class StaticKernel(metaclass=ABCMeta):
  """Base class of the static kernels (ksig/static/kernels.py:100-127)."""

  kind = None

  @property
  def param(self):
    raise NotImplementedError

  def fit(self, X, y=None):
    return self

  @staticmethod
  def _as_tensor(X):
    if isinstance(X, torch.Tensor):
      return X.to('cuda')
    return torch.as_tensor(np.asarray(X), device='cuda')

  def _validate_data(self, X):
    """Merges the last two axes when ``ndim > 2`` (ksig/static/kernels.py:125-127)."""
    if X.ndim > 2:
      X = X.reshape(X.shape[:-2] + (-1,))
    return X

  def __call__(self, X, Y=None, diag=False, return_on_gpu=False):
    """Static Gram ``[..., nX, nY]`` or its diagonal (ksig/static/kernels.py:71-97)."""
    X = self._validate_data(self._as_tensor(X))
    if diag:
      K = self._Kdiag(X)
    else:
      Y = self._validate_data(self._as_tensor(Y)) if Y is not None else None
      K = self._K(X, Y)
    return K if return_on_gpu else K.cpu().numpy()


class LinearKernel(StaticKernel):
  """``scale * <x, y>`` (ksig/static/kernels.py:134-166)."""

  kind = STATIC_LINEAR

  def __init__(self, scale: float = 1.):
    self.scale = utils.check_positive_value(scale, 'scale')

  @property
  def param(self):
    v = self.scale
    return float(v.detach()) if hasattr(v, 'detach') else float(v)

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    return self.scale * torch.einsum('...ij,...kj->...ik', X, Y)

  def _Kdiag(self, X):
    return self.scale * torch.sum(X * X, dim=-1)


class StationaryKernel(StaticKernel):
  """Stationary kernels with unit diagonal (ksig/static/kernels.py:214-242)."""

  def __init__(self, bandwidth: float = 1.) -> None:
    self.bandwidth = utils.check_positive_value(bandwidth, 'bandwidth')

  @property
  def param(self):
    v = self.bandwidth
    return float(v.detach()) if hasattr(v, 'detach') else float(v)

  def _Kdiag(self, X):
    return torch.ones((X.shape[0],), dtype=X.dtype, device=X.device)


class RBFKernel(StationaryKernel):
  """``exp(-|x-y|^2 / max(2 bandwidth^2, 1e-12))`` (ksig/static/kernels.py:245-260)."""

  kind = STATIC_RBF

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    xn = torch.sum(X * X, dim=-1)
    yn = torch.sum(Y * Y, dim=-1)
    d2 = xn[..., :, None] + yn[..., None, :] - 2 * torch.einsum(
        '...ij,...kj->...ik', X, Y)
    return torch.exp(-d2 / max(2 * self.bandwidth ** 2, utils._EPS))
