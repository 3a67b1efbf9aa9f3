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
from .._lib import (STATIC_LINEAR, STATIC_MATERN12, STATIC_MATERN32, STATIC_MATERN52,
                    STATIC_POLY, STATIC_RBF, STATIC_RQ)


def _f(v):
  return float(v.detach()) if hasattr(v, 'detach') else float(v)


def _sq_dist(X, Y):
  xn = torch.sum(X * X, dim=-1)
  yn = torch.sum(Y * Y, dim=-1)
  return xn[..., :, None] + yn[..., None, :] - 2 * torch.einsum('...ij,...kj->...ik', X, Y)


class StaticKernel(metaclass=ABCMeta):
  """Base class of the static kernels (ksig/static/kernels.py:100-127)."""

  kind = None

  @property
  def param(self):
    raise NotImplementedError

  @property
  def params(self):
    """The parameter list the fused kernels take for this kind (the
    KSIG_STATIC_* comments in include/ksig_b200.h)."""
    return (self.param,)

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


class PolynomialKernel(StaticKernel):
  """``scale * (<x, y> + gamma)^degree`` (ksig/static/kernels.py:169-203)."""

  kind = STATIC_POLY

  def __init__(self, degree: float = 3., gamma: float = 1., scale: float = 1.):
    self.degree = utils.check_positive_value(degree, 'degree')
    self.gamma = gamma
    self.scale = utils.check_positive_value(scale, 'scale')

  @property
  def param(self):
    return _f(self.degree)

  @property
  def params(self):
    return (_f(self.degree), _f(self.gamma), _f(self.scale))

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    return self.scale * torch.pow(torch.einsum('...ij,...kj->...ik', X, Y) + self.gamma,
                                  self.degree)

  def _Kdiag(self, X):
    return self.scale * torch.pow(torch.sum(X * X, dim=-1) + self.gamma, self.degree)


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


class Matern12Kernel(StationaryKernel):
  """``exp(-|x-y| / bandwidth)`` (ksig/static/kernels.py:263-277), with the
  distance between x and y.  The reference's ``euclid_dist``
  (ksig/utils.py:186-197) takes a stray ``self`` argument and returns the
  distances within its second argument instead; that is not reproduced."""

  kind = STATIC_MATERN12

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    D = torch.sqrt(torch.clamp(_sq_dist(X, Y), min=utils._EPS)) / max(self.bandwidth, utils._EPS)
    return torch.exp(-D)


class Matern32Kernel(StationaryKernel):
  """``(1 + D) exp(-D)``, ``D = sqrt(3) |x-y| / bandwidth``
  (ksig/static/kernels.py:280-296; distance as in :class:`Matern12Kernel`)."""

  kind = STATIC_MATERN32

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    D = (np.sqrt(3.) * torch.sqrt(torch.clamp(_sq_dist(X, Y), min=utils._EPS))
         / max(self.bandwidth, utils._EPS))
    return (1. + D) * torch.exp(-D)


class Matern52Kernel(StationaryKernel):
  """``(1 + D + D^2/3) exp(-D)``, ``D^2 = 5 |x-y|^2 / bandwidth^2``
  (ksig/static/kernels.py:299-316)."""

  kind = STATIC_MATERN52

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    E = 5 * _sq_dist(X, Y) / max(self.bandwidth ** 2, utils._EPS)
    D = torch.sqrt(torch.clamp(E, min=utils._EPS))
    return (1. + D + E / 3.) * torch.exp(-D)


class RationalQuadraticKernel(StationaryKernel):
  """``(1 + |x-y|^2 / (2 alpha bandwidth^2))^-alpha``
  (ksig/static/kernels.py:319-343)."""

  kind = STATIC_RQ

  def __init__(self, bandwidth: float = 1., alpha: float = 1.):
    super().__init__(bandwidth=bandwidth)
    self.alpha = utils.check_positive_value(alpha, 'alpha')

  @property
  def params(self):
    return (_f(self.bandwidth), _f(self.alpha))

  def _K(self, X, Y=None):
    Y = X if Y is None else Y
    E = _sq_dist(X, Y) / max(2 * self.alpha * self.bandwidth ** 2, utils._EPS)
    return torch.pow(1 + E, -self.alpha)
