"""Kernel-matrix precompute for precomputed-kernel SVMs.

Replaces ``PrecomputedSVCBase._precompute_kernel_mat``
(ksig/models/pre_base.py:88-142), which fills the matrix with a host loop
over ``batch_size x batch_size`` blocks, one kernel call and one
device-to-host copy per block.  Here a block row is one call (two in the
symmetric case: the diagonal block as a symmetric call, the rest of the
row to its right): the persistent pair sweep covers every pair of the row
block in one launch, the symmetric case evaluates only the upper triangle
and mirrors it on the device, and the assembled matrix crosses to the host
once.  For the signature kernels of this package the per-level diagonal
kernels that normalisation needs are computed once per call (one diagonal
pass per side), and every block normalises its levels with slices of them,
so the blocks equal the corresponding entries of the full matrix exactly as
in the reference, whose blocks each repeat the diagonal passes.
"""

from math import ceil
from typing import Callable, Optional

import numpy as np
import torch


def _rows(X, a, b):
  return X[a:b]


def _as_tensor(K):
  return K if isinstance(K, torch.Tensor) else torch.as_tensor(np.asarray(K))


def _level_path(kernel):
  """The kernel's per-level entry points when it is one of this package's
  level-based signature kernels (not the log-space alignment kernel)."""
  from . import kernels as Kmod
  return (isinstance(kernel, Kmod.SignatureKernel) and hasattr(kernel, '_levels'))


def _sub(S, a, b):
  from . import _engine as E
  return E.Seqs(S.data[a:b], None if S.lengths is None else S.lengths[a:b])


def _precompute_levels(kernel, X, X2, bs):
  """Block rows of per-level kernels, normalised with diagonals computed
  once per side."""
  from . import _engine as E
  from . import _lib as L
  from .kernels import _to_seqs
  Xs, _, _ = _to_seqs(X, kernel.n_features)
  Ys = Xs if X2 is None else _to_seqs(X2, kernel.n_features)[0]
  n, n2 = Xs.n, Ys.n
  norm = kernel.normalize
  dX = kernel._levels(Xs, None, L.PAIRS_DIAG) if norm else None
  dY = dX if (X2 is None or not norm) else kernel._levels(Ys, None, L.PAIRS_DIAG)
  out = torch.empty((n, n2), dtype=torch.float64, device=Xs.data.device)
  nb = ceil(n / bs)
  for i in range(nb):
    a, b = i * bs, min((i + 1) * bs, n)
    Xa = _sub(Xs, a, b)
    if X2 is None:
      lev = kernel._levels(Xa, None, L.PAIRS_UPPER)
      out[a:b, a:b] = E.normalize_levels(lev, L.PAIRS_UPPER, b - a, b - a, None, None,
                                         norm, torch.float64)
      if b < n:
        Yb = _sub(Xs, b, n)
        lev = kernel._levels(Xa, Yb, L.PAIRS_FULL)
        blk = E.normalize_levels(lev, L.PAIRS_FULL, b - a, n - b,
                                 None if dX is None else dX[:, a:b].contiguous(),
                                 None if dX is None else dX[:, b:n].contiguous(),
                                 norm, torch.float64)
        out[a:b, b:] = blk
        out[b:, a:b] = blk.transpose(0, 1)
    else:
      lev = kernel._levels(Xa, Ys, L.PAIRS_FULL)
      out[a:b] = E.normalize_levels(lev, L.PAIRS_FULL, b - a, n2,
                                    None if dX is None else dX[:, a:b].contiguous(),
                                    dY, norm, torch.float64)
  out_np = out.cpu().numpy()
  E.check_device_status()
  return out_np


def precompute_kernel_mat(kernel: Callable, X, X2=None,
                          batch_size: Optional[int] = None) -> np.ndarray:
  """The kernel matrix on the host as float64 ``[n, n]`` (``X2 is None``)
  or ``[n, n2]``.

  ``kernel`` is a ``ksig_b200`` kernel (or any callable with the
  ``kernel(X, Y, return_on_gpu=True)`` signature).  ``batch_size`` bounds
  the rows evaluated per call (memory), as the reference's argument does;
  ``None`` evaluates the whole matrix in one call.
  """
  if batch_size is not None and int(batch_size) <= 0:
    raise ValueError('batch_size must be positive')
  n = len(X)
  if batch_size is None or batch_size >= n:
    K = kernel(X, return_on_gpu=True) if X2 is None else kernel(X, X2, return_on_gpu=True)
    return _as_tensor(K).detach().to(torch.float64).cpu().numpy()
  bs = int(batch_size)
  if _level_path(kernel):
    return _precompute_levels(kernel, X, X2, bs)
  nb = ceil(n / bs)
  if X2 is None:
    out = None
    for i in range(nb):
      a, b = i * bs, min((i + 1) * bs, n)
      # Diagonal block: the symmetric call (upper triangle, mirrored);
      # the rest of the block row in one call, mirrored below.
      dg = _as_tensor(kernel(_rows(X, a, b), return_on_gpu=True)).detach().to(torch.float64)
      if out is None:
        out = torch.empty((n, n), dtype=torch.float64, device=dg.device)
      out[a:b, a:b] = dg
      if b < n:
        blk = _as_tensor(kernel(_rows(X, a, b), _rows(X, b, n), return_on_gpu=True))
        blk = blk.detach().to(torch.float64)
        out[a:b, b:] = blk
        out[b:, a:b] = blk.transpose(0, 1)
    return out.cpu().numpy()
  n2 = len(X2)
  out = None
  for i in range(nb):
    a, b = i * bs, min((i + 1) * bs, n)
    blk = _as_tensor(kernel(_rows(X, a, b), X2, return_on_gpu=True)).detach()
    blk = blk.to(torch.float64)
    if out is None:
      out = torch.empty((n, n2), dtype=torch.float64, device=blk.device)
    out[a:b] = blk
  return out.cpu().numpy()
