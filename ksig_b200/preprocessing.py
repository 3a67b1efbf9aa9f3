"""Sequence preprocessing on the device (ksig/preprocessing.py).

``SequenceTabulator`` and ``SequenceAugmentor`` keep the reference's
scikit-learn interface and results, computed with torch on the GPU so that
they feed the signature kernels without a host round trip.  With
``ragged=True`` the tabulator skips the interpolation to a common length and
returns a :class:`ksig_b200.Ragged` batch (padded data plus lengths): the
kernels here take ragged batches directly (no reference counterpart).
"""

from typing import List, Optional, Union

import numpy as np
import torch
from sklearn.base import BaseEstimator, TransformerMixin

from . import utils
from .kernels import Ragged


def _dev(x, dtype=None):
  t = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x))
  t = t.to('cuda')
  if dtype is not None:
    t = t.to(dtype)
  elif t.dtype not in (torch.float32, torch.float64):
    t = t.to(torch.float64)
  return t


def _interp_rows(x, n_out):
  """Linear interpolation of the rows of ``x [n, d]`` from ``linspace(0, 1,
  n)`` to ``linspace(0, 1, n_out)``, channel by channel (``np.interp``)."""
  n = x.shape[0]
  if n == 1:
    return x.expand(n_out, -1).clone()
  t = torch.linspace(0, 1, n_out, dtype=torch.float64, device=x.device)
  pos = t * (n - 1)
  lo = torch.clamp(torch.floor(pos).long(), 0, n - 2)
  w = (pos - lo.to(torch.float64)).to(x.dtype)[:, None]
  return x[lo] + w * (x[lo + 1] - x[lo])


def _as_list(X_seq):
  if isinstance(X_seq, (list, tuple)):
    return [_dev(x) for x in X_seq]
  X = _dev(X_seq)
  return [X[i] for i in range(X.shape[0])]


def _to_output(T, like):
  if isinstance(like, torch.Tensor) or isinstance(like, Ragged):
    return T
  if isinstance(like, (list, tuple)) and like and isinstance(like[0], torch.Tensor):
    return T
  return T.cpu().numpy() if isinstance(T, torch.Tensor) else T


class SequenceTabulator(BaseEstimator, TransformerMixin):
  """Tabulates sequences to a common length (ksig/preprocessing.py:15-67)."""

  def __init__(self, max_len: Optional[int] = None, ragged: bool = False):
    self.max_len = (utils.check_positive_value(max_len, 'max_len')
                    if max_len is not None else None)
    self.ragged = ragged

  def fit(self, X_seq, y=None) -> 'SequenceTabulator':
    max_seq_len = int(np.max([x.shape[0] for x in X_seq]))
    self.max_len_ = (min(self.max_len, max_seq_len) if self.max_len is not None
                     else max_seq_len)
    return self

  def transform(self, X_seq):
    """Interpolates every sequence channel-wise onto ``max_len_`` points
    when the lengths differ, a sequence holds NaNs or exceeds ``max_len_``
    (rows holding a NaN are dropped first); otherwise stacks them.  With
    ``ragged`` the sequences (NaN rows dropped) are returned as a Ragged
    batch instead of being interpolated, unless one exceeds ``max_len_``."""
    xs = _as_list(X_seq)
    lens = [x.shape[0] for x in xs]
    has_nan = any(bool(torch.isnan(x).any()) for x in xs)
    needs = has_nan or any(n != lens[0] for n in lens) or any(n > self.max_len_ for n in lens)
    if needs:
      xs = [x[torch.all(~torch.isnan(x), dim=-1)] for x in xs]
      if self.ragged and all(x.shape[0] <= self.max_len_ for x in xs):
        L = max(x.shape[0] for x in xs)
        data = torch.zeros((len(xs), L, xs[0].shape[1]), dtype=xs[0].dtype, device='cuda')
        for i, x in enumerate(xs):
          data[i, :x.shape[0]] = x
        return Ragged(data, torch.tensor([x.shape[0] for x in xs], dtype=torch.int32,
                                         device='cuda'))
      xs = [_interp_rows(x, self.max_len_) for x in xs]
    return _to_output(torch.stack(xs, dim=0), X_seq)


class SequenceAugmentor(BaseEstimator, TransformerMixin):
  """Normalisation, lead-lag, time and basepoint augmentation
  (ksig/preprocessing.py:72-136)."""

  def __init__(self, add_time: bool = True, lead_lag: bool = True,
               basepoint: bool = True, normalize: bool = True,
               max_time: float = 1., max_len: Optional[int] = None):
    self.add_time = add_time
    self.lead_lag = lead_lag
    self.basepoint = basepoint
    self.normalize = normalize
    self.max_time = max_time
    self.max_len = max_len

  def fit(self, X_seq, y=None) -> 'SequenceAugmentor':
    if self.normalize:
      self.scale_ = _dev(X_seq).max()
    return self

  def transform(self, X_seq):
    """Same steps and order as the reference; the input is not modified
    (the reference divides it in place)."""
    X = _dev(X_seq)
    if self.normalize:
      X = X / self.scale_.to(X.dtype)
    if self.lead_lag:
      X = torch.repeat_interleave(X, 2, dim=1)
      X = torch.cat((X[:, 1:], X[:, :-1]), dim=-1)
    if self.add_time and self.max_time > 1e-6:
      t = torch.linspace(0., self.max_time, X.shape[1], dtype=torch.float64,
                         device=X.device).to(X.dtype)
      X = torch.cat((t[None, :, None].expand(X.shape[0], -1, 1), X), dim=-1)
    if self.basepoint:
      X = torch.cat((torch.zeros_like(X[:, :1]), X), dim=1)
    if self.max_len is not None and X.shape[1] > self.max_len:
      X = torch.stack([_interp_rows(x, self.max_len) for x in X], dim=0)
    return _to_output(X, X_seq)
