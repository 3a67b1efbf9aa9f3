"""Signature kernels with KSig's callable API, computed by sm_100a kernels.

``SignatureKernel`` and ``SignaturePDEKernel`` keep the constructor and call
semantics of ``ksig.kernels`` (ksig/kernels.py:25-256)::

    K = SignatureKernel(n_levels=5, order=1, difference=True, normalize=True,
                        n_features=None, static_kernel=RBFKernel(1.0))
    K(X)                 # [nX, nX]
    K(X, Y)              # [nX, nY]
    K(X, diag=True)      # [nX]
    K(X, Y, return_on_gpu=True)   # torch CUDA tensor instead of NumPy

``X`` / ``Y`` may be NumPy arrays, PyTorch tensors (CPU or CUDA) of shape
``[n, L, d]`` (or ``[n, L*d]`` with ``n_features``), or a list of ``[L_i, d]``
arrays of different lengths (ragged; no reference counterpart — the result
equals the reference on the edge-padded dense array).  The arithmetic runs
in the input dtype (float32 -> FP32 kernels with FP64 reductions, float64 ->
FP64).  Torch inputs that require grad (and an RBF ``bandwidth`` given as a
tensor that requires grad) are differentiated through a hand-written
adjoint.
"""

import warnings
from typing import Optional

import numpy as np
import torch

from . import _autograd as AG
from . import _engine as E
from . import _lib as L
from . import static as static_mod
from . import utils
from .static.kernels import StaticKernel


class Ragged:
  """A ragged batch as one dense padded tensor plus per-sequence lengths.

  ``data`` is ``[n, L, d]`` (points past ``lengths[i]`` are ignored, which
  equals the reference on the edge-padded array) and ``lengths`` ``[n]``.
  Unlike a Python list it costs no per-sequence copies, keeps fixed device
  buffers (so a call on it can be captured in a CUDA graph) and, when
  ``data`` requires grad, takes gradients directly.  No reference
  counterpart.
  """

  __slots__ = ('data', 'lengths')

  def __init__(self, data, lengths):
    data = torch.as_tensor(data)
    lengths = torch.as_tensor(lengths)
    if data.ndim != 3:
      raise ValueError('Ragged data must be [n, L, d]')
    if lengths.ndim != 1 or lengths.shape[0] != data.shape[0]:
      raise ValueError('Ragged lengths must be [n]')
    self.data = data
    self.lengths = lengths

  def __len__(self):
    return self.data.shape[0]


def _is_ragged(X):
  return isinstance(X, (list, tuple))


def _to_seqs(X, n_features, reset_obj=None):
  """Validates and moves a batch of sequences to the device.

  Mirrors ``SignatureBase._validate_data`` (ksig/kernels.py:56-90) for dense
  inputs; ragged inputs (lists) are padded and carry their lengths.
  Returns (Seqs, was_torch, requires_grad_tensor_or_None).
  """
  if isinstance(X, Ragged):
    data = X.data
    if n_features is not None and data.shape[-1] != n_features:
      raise ValueError(
          'Number of features in `X` does not match saved `n_features` param.')
    if data.dtype not in (torch.float32, torch.float64):
      data = data.to(torch.float64)
    lengths = X.lengths.to(device='cuda', dtype=torch.int32)
    # Host-side range check, skipped while a CUDA graph is being captured
    # (it would synchronise); the packing kernel checks the lengths on the
    # device as well.
    if (not torch.cuda.is_current_stream_capturing() and int(lengths.numel()) and
        (bool((lengths < 0).any()) or bool((lengths > data.shape[1]).any()))):
      raise ValueError('Ragged lengths must lie in [0, L]')
    lengths = lengths.clamp_min(1)
    grad_src = data if data.requires_grad else None
    Xd = data.detach().to('cuda').contiguous()
    return E.Seqs(Xd, lengths), False, grad_src
  if _is_ragged(X):
    seqs = [s if isinstance(s, torch.Tensor) else torch.as_tensor(np.asarray(s))
            for s in X]
    if not seqs:
      raise ValueError('empty sequence list')
    seqs = [s.reshape(s.shape[0], -1) if s.ndim != 2 else s for s in seqs]
    d = seqs[0].shape[-1]
    if any(s.shape[-1] != d for s in seqs):
      raise ValueError('all sequences must have the same number of features')
    if n_features is not None and d != n_features:
      raise ValueError(
          'Number of features in `X` does not match saved `n_features` param.')
    dtype = seqs[0].dtype if seqs[0].dtype in (torch.float32, torch.float64) \
        else torch.float64
    lens = [max(int(s.shape[0]), 1) for s in seqs]
    Lmax = max(lens)
    lengths = torch.tensor(lens, dtype=torch.int32, device='cuda')
    if any(s.requires_grad for s in seqs):
      # Differentiable padding: gradients flow back to the list entries.
      padded = torch.nn.utils.rnn.pad_sequence(
          [s.to(device='cuda', dtype=dtype) if s.shape[0] > 0
           else torch.zeros((1, d), dtype=dtype, device='cuda') for s in seqs],
          batch_first=True)
      return E.Seqs(padded.detach().contiguous(), lengths), False, padded
    if all(not s.is_cuda for s in seqs):
      # Host sequences: padded on the host, one host-to-device copy.
      host = np.zeros((len(seqs), Lmax, d),
                      dtype=np.float64 if dtype == torch.float64 else np.float32)
      for i, s in enumerate(seqs):
        if s.shape[0] > 0:
          host[i, :s.shape[0]] = s.detach().numpy()
      data = torch.from_numpy(host).to('cuda', non_blocking=False)
    else:
      # Device sequences: one padding kernel, no per-sequence copies.
      data = torch.nn.utils.rnn.pad_sequence(
          [s.to(device='cuda', dtype=dtype) if s.shape[0] > 0
           else torch.zeros((1, d), dtype=dtype, device='cuda') for s in seqs],
          batch_first=True)
      if data.shape[1] < Lmax:
        data = torch.nn.functional.pad(data, (0, 0, 0, Lmax - data.shape[1]))
    return E.Seqs(data.contiguous(), lengths), False, None
  was_torch = isinstance(X, torch.Tensor)
  if not was_torch:
    X = torch.as_tensor(np.asarray(X))
  if X.ndim == 2:
    if n_features is None:
      warnings.warn('`X` has ndim==2. Assuming inputs are univariate time '
                    'series. Recommend passing an `n_features` parameter '
                    'during init when using flattened arrays of ndim==2.')
      n_features = 1
  elif X.ndim == 3:
    if n_features is None:
      n_features = X.shape[-1]
    elif X.shape[-1] != n_features:
      raise ValueError(
          'Number of features in `X` does not match saved `n_features` param.')
  else:
    raise ValueError(
        'Only input sequence arrays with ndim==2 or ndim==3 are supported.')
  X = X.reshape([X.shape[0], -1, n_features])
  if X.dtype not in (torch.float32, torch.float64):
    X = X.to(torch.float64)
  grad_src = X if (was_torch and X.requires_grad) else None
  Xd = X.detach().to('cuda').contiguous()
  return E.Seqs(Xd), was_torch, grad_src


class SignatureBase:
  """Shared parameters and validation (ksig/kernels.py:25-90)."""

  def __init__(self, n_levels: int = 5, order: int = 1,
               difference: bool = True, normalize: bool = True,
               n_features: Optional[int] = None):
    self.n_levels = utils.check_positive_value(n_levels, 'n_levels')
    self.order = (self.n_levels if order <= 0 or order >= self.n_levels
                  else order)
    self.normalize = normalize
    self.difference = difference
    self.n_features = (utils.check_positive_value(n_features, 'n_features')
                       if n_features is not None else None)

  def fit(self, X, y=None):
    return self

  def _static(self):
    """(kind, parameter): one float for RBF / linear, the parameter tuple
    for the other static kernels (fused into the Gram epilogue alike)."""
    sk = self.static_kernel
    if not isinstance(sk, StaticKernel) or sk.kind is None:
      raise ValueError('static_kernel must be one of the kernels of '
                       'ksig_b200.static.kernels')
    if sk.kind in (L.STATIC_RBF, L.STATIC_LINEAR):
      return sk.kind, sk.param
    return sk.kind, tuple(sk.params)

  def __call__(self, X, Y=None, diag: bool = False,
               return_on_gpu: bool = False):
    """Kernel matrix ``K(X, Y)``, ``K(X, X)`` or its diagonal
    (``Kernel.__call__``, ksig/static/kernels.py:71-97)."""
    if not torch.cuda.is_available():
      raise RuntimeError('ksig_b200 needs a CUDA device (no CPU fallback)')
    Xs, _, gx = _to_seqs(X, self.n_features)
    Ys, gy = None, None
    if not diag and Y is not None:
      Ys, _, gy = _to_seqs(Y, self.n_features)
    if diag:
      K = self._Kdiag(Xs)
    elif torch.is_grad_enabled() and (gx is not None or gy is not None or
                                      self._param_requires_grad()):
      K = self._K_autograd(X if gx is not None else None, Xs, gx,
                           Ys, gy, Y is None)
    else:
      K = self._K(Xs, Ys)
    if return_on_gpu:
      return K
    if K.requires_grad:
      return K
    out = K.detach().cpu().numpy()
    E.check_device_status()  # the copy above has synchronised already
    return out

  def _param_tensor(self):
    sk = self.static_kernel
    p = getattr(sk, 'bandwidth', None)
    if p is None:
      p = getattr(sk, 'scale', None)
    return p if isinstance(p, torch.Tensor) else None

  def _param_requires_grad(self):
    p = self._param_tensor()
    return p is not None and p.requires_grad

  def _levels_bwd(self, Xs, Ys, mode, grad_levels, want_dparam):
    raise NotImplementedError(
        f'gradients are not available for {type(self).__name__}')

  def _split_pass(self):
    """(forward, adjoint) of the split gradient pass for K(X, Y), or None
    where it does not apply."""
    return None

  def _K_autograd(self, Xin, Xs, gx, Ys, gy, sym):
    """Differentiable K(X, Y) / K(X) through the hand-written adjoint."""
    kind, param = self._static()
    if kind not in (L.STATIC_RBF, L.STATIC_LINEAR):
      raise NotImplementedError(
          'gradients are available with the RBF and linear static kernels')
    pt = self._param_tensor()
    spec = dict(Xs=Xs, Ys=Ys, normalize=self.normalize, kind=kind,
                param=float(param), levels_fn=self._levels,
                bwd_fn=self._levels_bwd, rec_fn=self._split_pass(),
                param_dtype=pt.dtype if pt is not None else torch.float64,
                param_device=pt.device if pt is not None else 'cpu',
                const_level0=not isinstance(self, SignaturePDEKernel))
    if sym:
      gy = None
    return AG.SigKernelFn.apply(gx, gy, pt if (pt is not None and pt.requires_grad)
                                else None, spec)


class SignatureKernel(SignatureBase):
  """Full-rank truncated signature kernel (ksig/kernels.py:97-214)."""

  def __init__(self, n_levels: int = 5, order: int = 1,
               difference: bool = True, normalize: bool = True,
               n_features: Optional[int] = None,
               static_kernel: Optional[StaticKernel] = None):
    super().__init__(n_levels=n_levels, order=order, difference=difference,
                     normalize=normalize, n_features=n_features)
    self.static_kernel = static_kernel or static_mod.kernels.RBFKernel()

  # -- level kernels ------------------------------------------------------
  def _levels(self, Xs, Ys, mode):
    kind, param = self._static()
    return E.sig_levels(Xs, Ys, mode, self.n_levels, self.order,
                        self.difference, kind, param)

  def _levels_bwd(self, Xs, Ys, mode, grad_levels, want_dparam):
    kind, param = self._static()
    return E.sig_levels_bwd(Xs, Ys, mode, self.n_levels, self.order, kind,
                            param, grad_levels, want_dparam=want_dparam)

  def _split_pass(self):
    """Order 1 with differencing: the autograd forward runs the forward
    pass of the adjoint kernel and keeps its per-pair records (when they fit
    the memory budget of ``_engine.rec_budget_bytes``), so the backward runs
    only the adjoint pass."""
    if self.order != 1 or self.n_levels < 2 or not self.difference:
      return None
    kind, param = self._static()

    def fwd(Xs, Ys):
      return E.sig_levels_rec(Xs, Ys, self.n_levels, 1, kind, param)

    def bwd(Xs, Ys, grad_levels, want_dparam, ws):
      return E.sig_levels_bwd_rec(Xs, Ys, self.n_levels, 1, kind, param,
                                  grad_levels, ws, want_dparam=want_dparam)
    return fwd, bwd

  def _Kdiag(self, Xs):
    """ksig/kernels.py:166-178: ones when normalising."""
    if self.normalize:
      return torch.full((Xs.n,), 1., dtype=torch.float64,
                        device=Xs.data.device)
    lev = self._levels(Xs, None, L.PAIRS_DIAG)
    return lev.sum(dim=0).to(Xs.data.dtype)

  def _K(self, Xs, Ys=None):
    """ksig/kernels.py:180-214 (levels -> per-level normalisation -> mean)."""
    out_dtype = Xs.data.dtype
    if Ys is None:
      lev = self._levels(Xs, None, L.PAIRS_UPPER)
      return E.normalize_levels(lev, L.PAIRS_UPPER, Xs.n, Xs.n, None, None,
                                self.normalize, out_dtype)
    lev = self._levels(Xs, Ys, L.PAIRS_FULL)
    dx = dy = None
    if self.normalize:
      dx = self._levels(Xs, None, L.PAIRS_DIAG)
      dy = self._levels(Ys, None, L.PAIRS_DIAG)
    return E.normalize_levels(lev, L.PAIRS_FULL, Xs.n, Ys.n, dx, dy,
                              self.normalize, out_dtype)


class SignaturePDEKernel(SignatureKernel):
  """Signature-PDE kernel (ksig/kernels.py:218-256).

  ``dyadic_order`` (no reference counterpart; default 0 = the reference
  scheme) refines every cell of the Goursat grid into 2^k x 2^k cells.
  """

  def __init__(self, difference: bool = True, normalize: bool = True,
               n_features: Optional[int] = None,
               static_kernel: Optional[StaticKernel] = None,
               dyadic_order: int = 0):
    self.difference = difference
    self.normalize = normalize
    self.n_features = (utils.check_positive_value(n_features, 'n_features')
                       if n_features is not None else None)
    self.static_kernel = static_kernel or static_mod.kernels.RBFKernel()
    if int(dyadic_order) < 0:
      raise ValueError('dyadic_order must be non-negative')
    self.dyadic_order = int(dyadic_order)

  def _levels(self, Xs, Ys, mode):
    kind, param = self._static()
    v = E.pde_values(Xs, Ys, mode, self.dyadic_order, self.difference, kind,
                     param)
    return v[None, :]

  def _levels_bwd(self, Xs, Ys, mode, grad_levels, want_dparam):
    kind, param = self._static()
    return E.pde_values_bwd(Xs, Ys, mode, self.dyadic_order, kind, param,
                            grad_levels[0], want_dparam=want_dparam)

  def _split_pass(self):
    return None  # the split gradient pass is the DP adjoint's


class GlobalAlignmentKernel(SignatureBase):
  """Global alignment kernel (ksig/kernels.py:366-409), always normalised.

  ``K(x, y) = exp(logGA(x, y) - (logGA(x, x) + logGA(y, y)) / 2)`` with the
  log-space alignment recursion of ksig/algorithms.py:453-559 run by the
  persistent skewed sweep (``ksig_global_align_kern``); the normalisation
  follows the log-space branch of ksig/kernels.py:190-206 and
  ``K(X, diag=True)`` returns ones.  Static kernels: RBF and linear.
  """

  def __init__(self, n_features: Optional[int] = None,
               static_kernel: Optional[StaticKernel] = None):
    self.n_features = (utils.check_positive_value(n_features, 'n_features')
                       if n_features is not None else None)
    self.static_kernel = static_kernel or static_mod.kernels.RBFKernel()

  @property
  def normalize(self):
    return True

  @property
  def is_log_space(self):
    return True

  def _static(self):
    kind, param = super()._static()
    if kind not in (L.STATIC_RBF, L.STATIC_LINEAR):
      raise ValueError('GlobalAlignmentKernel supports the RBF and linear '
                       'static kernels')
    return kind, param

  def __call__(self, X, Y=None, diag: bool = False,
               return_on_gpu: bool = False):
    if not torch.cuda.is_available():
      raise RuntimeError('ksig_b200 needs a CUDA device (no CPU fallback)')
    Xs, _, _ = _to_seqs(X, self.n_features)
    if diag:
      K = torch.ones((Xs.n,), dtype=torch.float64, device=Xs.data.device)
    else:
      kind, param = self._static()
      if Y is None:
        up = E.ga_values(Xs, None, L.PAIRS_UPPER, kind, param)
        n = Xs.n
        iu = torch.triu_indices(n, n, device=up.device)
        lk = torch.empty((n, n), dtype=torch.float64, device=up.device)
        lk[iu[0], iu[1]] = up
        lk[iu[1], iu[0]] = up
        d = torch.diagonal(lk)
        lk = lk - 0.5 * (d[:, None] + d[None, :])
      else:
        Ys, _, _ = _to_seqs(Y, self.n_features)
        lk = E.ga_values(Xs, Ys, L.PAIRS_FULL, kind, param).reshape(Xs.n, Ys.n)
        dx = E.ga_values(Xs, None, L.PAIRS_DIAG, kind, param)
        dy = E.ga_values(Ys, None, L.PAIRS_DIAG, kind, param)
        lk = lk - 0.5 * (dx[:, None] + dy[None, :])
      K = torch.exp(lk).to(Xs.data.dtype)
    if return_on_gpu:
      return K
    out = K.detach().cpu().numpy()
    E.check_device_status()
    return out
