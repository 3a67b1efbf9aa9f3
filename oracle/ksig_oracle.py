"""FP64 CPU oracle for the signature-kernel hot path (test infrastructure).

This module is the checker, not the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it.  It restates, in NumPy float64, the algorithms of KSig 1.0.0
(tgcsaba/KSig) on the path that ``ksig_b200`` implements in CUDA:

* static Gram: ``RBFKernel._K`` (ksig/static/kernels.py:248-260) through
  ``squared_euclid_dist`` (ksig/utils.py:138-157), and ``LinearKernel._K``
  (ksig/static/kernels.py:145-155);
* second difference ``cp.diff(cp.diff(M, -2), -1)``
  (ksig/algorithms.py:63-64, 105-106, 420-421);
* truncated DP signature kernel, first order (Alg. 3,
  ksig/algorithms.py:47-85) and higher order (Alg. 6,
  ksig/algorithms.py:88-140), built on ``multi_cumsum``
  (ksig/utils.py:63-90);
* Goursat PDE scheme (ksig/algorithms.py:344-399, update at :384-385),
  extended with dyadic refinement (``dyadic_order`` > 0 refines every cell
  into 2^k x 2^k sub-cells carrying ``q / 4^k``; order 0 is the reference);
* per-level normalisation and level mean of ``SignatureKernel._K``
  (ksig/kernels.py:180-214) with ``robust_sqrt`` (ksig/utils.py:173-182)
  and ``_EPS = 1e-12`` (ksig/utils.py:16).

Pinning: the functions here are checked against outputs of the reference
package itself (run on the CPU through a NumPy stand-in for CuPy and the
Numba CUDA simulator), committed under ``tests/golden/`` with the script that
produced them.  Dyadic orders > 0 and ragged batches have no reference
counterpart; the latter are pinned through the reference's padding
invariance (edge-repeating a sequence leaves both kernels unchanged).

Sequences may be given as a dense array ``[n, L, d]`` or as a list of
``[L_i, d]`` arrays of different lengths (ragged).
"""

from __future__ import annotations

import numpy as np

EPS = 1e-12  # ksig/utils.py:16

__all__ = [
    'EPS', 'static_gram', 'second_difference', 'multi_cumsum_exclusive',
    'sig_levels_first_order', 'sig_levels_higher_order', 'sig_levels',
    'sig_pde', 'signature_kernel', 'signature_pde_kernel', 'as_seq_list',
    'normalize_levels', 'ga_log', 'global_align_kernel',
]


# ----------------------------------------------------------------------------
# Static kernels.
# ----------------------------------------------------------------------------

def static_gram(X, Y, kind='rbf', param=1.0):
  """Static Gram between point sets ``X [..., m, d]`` and ``Y [..., n, d]``.

  RBF follows ksig/static/kernels.py:258-260: ``exp(-D2 / max(2 s^2, 1e-12))``
  with ``D2 = |x|^2 + |y|^2 - 2 x.y`` (ksig/utils.py:149-156), no clamp of
  negative D2.  Linear follows ksig/static/kernels.py:155: ``scale * x.y``.
  """
  X = np.asarray(X, dtype=np.float64)
  Y = np.asarray(Y, dtype=np.float64)
  xy = np.einsum('...ij,...kj->...ik', X, Y)
  if kind == 'rbf':
    xn = np.sum(np.square(X), axis=-1)
    yn = np.sum(np.square(Y), axis=-1)
    d2 = xn[..., :, None] + yn[..., None, :] - 2 * xy
    return np.exp(-d2 / max(2 * float(param) ** 2, EPS))
  if kind == 'linear':
    return float(param) * xy
  if kind == 'poly':  # ksig/static/kernels.py:183-194, param = (degree, gamma, scale)
    degree, gamma, scale = param
    return scale * np.power(xy + gamma, degree)
  xn = np.sum(np.square(X), axis=-1)
  yn = np.sum(np.square(Y), axis=-1)
  d2 = xn[..., :, None] + yn[..., None, :] - 2 * xy
  if kind in ('matern12', 'matern32'):
    # ksig/static/kernels.py:263-296 with the distance between x and y
    # (robust_sqrt, ksig/utils.py:173-182).  The reference's euclid_dist
    # (ksig/utils.py:186-197) takes a stray `self` argument and measures
    # within its second set instead; this restates the intended kernel.
    c = np.sqrt(3.) if kind == 'matern32' else 1.0
    D = c * np.sqrt(np.maximum(d2, EPS)) / max(float(param), EPS)
    return np.exp(-D) if kind == 'matern12' else (1. + D) * np.exp(-D)
  if kind == 'matern52':  # ksig/static/kernels.py:299-316
    E = 5 * d2 / max(float(param) ** 2, EPS)
    D = np.sqrt(np.maximum(E, EPS))
    return (1. + D + E / 3.) * np.exp(-D)
  if kind == 'rq':  # ksig/static/kernels.py:319-343, param = (bandwidth, alpha)
    bw, alpha = param
    E = d2 / max(2 * alpha * bw ** 2, EPS)
    return np.power(1 + E, -alpha)
  raise ValueError(f'unknown static kernel {kind!r}')


def second_difference(M):
  """``cp.diff(cp.diff(M, axis=-2), axis=-1)`` (ksig/algorithms.py:64)."""
  return np.diff(np.diff(M, axis=-2), axis=-1)


def multi_cumsum_exclusive(M, axis):
  """Exclusive cumulative sum over ``axis`` (ksig/utils.py:63-90).

  Slices off the last entry along each axis, cumsums along each axis in
  turn and zero-pads at the front, exactly as the reference does.
  """
  axis = [axis] if np.isscalar(axis) else list(axis)
  nd = M.ndim
  axis = [nd + a if a < 0 else a for a in axis]
  sl = tuple(slice(-1) if a in axis else slice(None) for a in range(nd))
  M = M[sl]
  for a in axis:
    M = np.cumsum(M, axis=a)
  pads = tuple((1, 0) if a in axis else (0, 0) for a in range(nd))
  return np.pad(M, pads)


# ----------------------------------------------------------------------------
# DP signature kernel (levels).
# ----------------------------------------------------------------------------

def sig_levels_first_order(Z, n_levels):
  """Per-level kernels ``[n_levels+1, ...]`` of Alg. 3 on increments ``Z``.

  ``Z`` is the (already differenced) static-kernel array ``[..., lx, ly]``.
  Follows ksig/algorithms.py:65-85 with ``return_levels=True``: level 0 is
  ones, level 1 is ``sum(Z)``, level k is ``sum(Z * excl2d(R_{k-1}))``.
  """
  K = [np.ones(Z.shape[:-2]), np.sum(Z, axis=(-2, -1))]
  R = np.copy(Z)
  for _ in range(1, n_levels):
    R = Z * multi_cumsum_exclusive(R, axis=(-2, -1))
    K.append(np.sum(R, axis=(-2, -1)))
  return np.stack(K, axis=0)


def sig_levels_higher_order(Z, n_levels, order):
  """Per-level kernels of Alg. 6 (ksig/algorithms.py:105-140)."""
  K = [np.ones(Z.shape[:-2]), np.sum(Z, axis=(-2, -1))]
  R = np.copy(Z)[None, None, ...]
  for i in range(1, n_levels):
    d = min(i + 1, order)
    R_next = np.empty((d, d) + Z.shape, dtype=Z.dtype)
    R_next[0, 0] = Z * multi_cumsum_exclusive(
        np.sum(R, axis=(0, 1)), axis=(-2, -1))
    for r in range(1, d):
      R_next[0, r] = 1. / (r + 1) * Z * multi_cumsum_exclusive(
          np.sum(R[:, r - 1], axis=0), axis=-2)
      R_next[r, 0] = 1. / (r + 1) * Z * multi_cumsum_exclusive(
          np.sum(R[r - 1, :], axis=0), axis=-1)
      for s in range(1, d):
        R_next[r, s] = 1. / ((r + 1) * (s + 1)) * Z * R[r - 1, s - 1]
    R = R_next
    K.append(np.sum(R, axis=(0, 1, -2, -1)))
  return np.stack(K, axis=0)


def clamp_order(n_levels, order):
  """Order clamp of ksig/algorithms.py:37 and ksig/kernels.py:49-50."""
  return n_levels if order <= 0 or order >= n_levels else order


def sig_levels(Z, n_levels, order=1):
  """Dispatch of ``signature_kern`` (ksig/algorithms.py:37-44)."""
  order = clamp_order(n_levels, order)
  if order == 1:
    return sig_levels_first_order(Z, n_levels)
  return sig_levels_higher_order(Z, n_levels, order)


# ----------------------------------------------------------------------------
# Goursat PDE.
# ----------------------------------------------------------------------------

def sig_pde(Z, dyadic_order=0):
  """Goursat-PDE signature kernel of ksig/algorithms.py:344-399.

  ``Z [..., lx, ly]`` holds the cell increments.  With refinement ``k`` each
  cell becomes ``2^k x 2^k`` cells with increment ``q = Z / 4^k``.  The
  scheme (ksig/algorithms.py:384-385) with boundary value 1 (:380-383):
  ``K[i+1,j+1] = (K[i,j+1] + K[i+1,j]) (1 + q/2 + q^2/12) - K[i,j] (1 - q^2/12)``;
  the result is the far corner.  Evaluated along antidiagonals, vectorised
  over the leading (pair) axes.
  """
  Z = np.asarray(Z, dtype=np.float64)
  f = 2 ** int(dyadic_order)
  if f > 1:
    Z = np.repeat(np.repeat(Z, f, axis=-2), f, axis=-1) / float(f * f)
  lead = Z.shape[:-2]
  lx, ly = Z.shape[-2:]
  if lx == 0 or ly == 0:
    return np.ones(lead)
  A = 1. + 0.5 * Z + (1. / 12) * Z ** 2
  B = 1. - (1. / 12) * Z ** 2
  K = np.ones(lead + (lx + 1, ly + 1))
  for s in range(lx + ly - 1):
    i = np.arange(max(0, s - ly + 1), min(s, lx - 1) + 1)
    j = s - i
    K[..., i + 1, j + 1] = ((K[..., i, j + 1] + K[..., i + 1, j]) * A[..., i, j]
                            - K[..., i, j] * B[..., i, j])
  return K[..., lx, ly]


# ----------------------------------------------------------------------------
# Sequence-kernel front ends (normalisation of ksig/kernels.py:180-214).
# ----------------------------------------------------------------------------

def as_seq_list(X):
  """Returns a list of ``[L_i, d]`` float64 arrays from dense or ragged X."""
  if isinstance(X, (list, tuple)):
    return [np.asarray(x, dtype=np.float64) for x in X]
  X = np.asarray(X, dtype=np.float64)
  if X.ndim != 3:
    raise ValueError('expected [n, L, d] or a list of [L_i, d]')
  return [X[i] for i in range(X.shape[0])]


def _pair_levels(x, y, fn, kind, param, difference):
  M = static_gram(x, y, kind, param)
  Z = second_difference(M) if difference else M
  return fn(Z)


def _gram_levels(Xs, Ys, fn, kind, param, difference, chunk=16):
  """Per-pair level arrays ``[..., nX, nY]`` over all pairs.

  Equal-length blocks are evaluated together (as the reference does with
  its ``[nX, nY, LX, LY]`` array), chunked ``chunk x chunk`` like the
  blocked precompute of ksig/models/pre_base.py:101-141.
  """
  nX, nY = len(Xs), len(Ys)
  out = None
  for a0 in range(0, nX, chunk):
    for b0 in range(0, nY, chunk):
      xa = Xs[a0:a0 + chunk]
      yb = Ys[b0:b0 + chunk]
      if len({x.shape for x in xa}) == 1 and len({y.shape for y in yb}) == 1:
        Xa = np.stack(xa)[:, None]
        Yb = np.stack(yb)[None]
        res = _pair_levels(Xa, Yb, fn, kind, param, difference)
        if out is None:
          out = np.zeros(res.shape[:-2] + (nX, nY))
        out[..., a0:a0 + len(xa), b0:b0 + len(yb)] = res
      else:
        for ia, x in enumerate(xa):
          for ib, y in enumerate(yb):
            res = _pair_levels(x, y, fn, kind, param, difference)
            if out is None:
              out = np.zeros(np.shape(res) + (nX, nY))
            out[..., a0 + ia, b0 + ib] = res
  return out


def _diag_levels(Xs, fn, kind, param, difference):
  outs = [_pair_levels(x, x, fn, kind, param, difference) for x in Xs]
  return np.stack(outs, axis=-1)


def normalize_levels(K, Kx, Ky):
  """``K / (max(robust_sqrt(Kx), eps) outer max(robust_sqrt(Ky), eps))``
  per level (ksig/kernels.py:197-207, ksig/utils.py:173-182), then the mean
  over levels when a level axis is present (ksig/kernels.py:212-213)."""
  sx = np.maximum(np.sqrt(np.maximum(Kx, EPS)), EPS)
  sy = np.maximum(np.sqrt(np.maximum(Ky, EPS)), EPS)
  K = K / (sx[..., :, None] * sy[..., None, :])
  if K.ndim == 3:
    K = np.mean(K, axis=0)
  return K


def _front(X, Y, diag, normalize, fn, kind, param, difference):
  Xs = as_seq_list(X)
  if diag:
    if normalize:
      return np.full((len(Xs),), 1.)  # ksig/kernels.py:175-176
    d = _diag_levels(Xs, fn, kind, param, difference)
    return d.sum(axis=0) if d.ndim == 2 else d
  Ys = Xs if Y is None else as_seq_list(Y)
  K = _gram_levels(Xs, Ys, fn, kind, param, difference)
  if normalize:
    if Y is None:
      Kd = np.einsum('...ii->...i', K)
      return normalize_levels(K, Kd, Kd)
    Kx = _diag_levels(Xs, fn, kind, param, difference)
    Ky = _diag_levels(Ys, fn, kind, param, difference)
    return normalize_levels(K, Kx, Ky)
  return K.sum(axis=0) if K.ndim == 3 else K


def signature_kernel(X, Y=None, diag=False, n_levels=5, order=1,
                     difference=True, normalize=True, kind='rbf', param=1.0,
                     return_levels=False):
  """FP64 ``SignatureKernel(...)(X, Y, diag)`` (ksig/kernels.py:97-214).

  With ``return_levels`` the un-normalised per-level array
  ``[n_levels+1, nX, nY]`` is returned instead (``signature_kern`` with
  ``return_levels=True``, ksig/algorithms.py:22-44).
  """
  fn = lambda Z: sig_levels(Z, n_levels, order)  # noqa: E731
  if return_levels:
    Xs = as_seq_list(X)
    Ys = Xs if Y is None else as_seq_list(Y)
    return _gram_levels(Xs, Ys, fn, kind, param, difference)
  return _front(X, Y, diag, normalize, fn, kind, param, difference)


def signature_pde_kernel(X, Y=None, diag=False, difference=True,
                         normalize=True, kind='rbf', param=1.0,
                         dyadic_order=0):
  """FP64 ``SignaturePDEKernel(...)(X, Y, diag)`` (ksig/kernels.py:218-256).

  Note: the reference's ``diag=True`` with ``normalize=True`` returns ones
  (inherited ``SignatureKernel._Kdiag``, ksig/kernels.py:175-176).
  """
  fn = lambda Z: sig_pde(Z, dyadic_order)  # noqa: E731
  return _front(X, Y, diag, normalize, fn, kind, param, difference)


# ----------------------------------------------------------------------------
# Global alignment kernel.
# ----------------------------------------------------------------------------

def ga_log(M):
  """Log global-alignment value of one pair from its static Gram ``M
  [lx, ly]`` (ksig/algorithms.py:513-559 and the antidiagonal kernel
  :453-510): ``M' = M / (2 - M)``, ``logM = log(max(M', 1e-12))``,
  ``logK[i,j] = logM[i,j] + logsumexp(logK[i-1,j], logK[i,j-1],
  logK[i-1,j-1])`` with ``logK[-1,-1] = 0`` and ``-inf`` elsewhere on the
  boundary; returns ``logK[lx-1, ly-1]``."""
  M = np.asarray(M, dtype=np.float64)
  logM = np.log(np.maximum(M / (2. - M), EPS))
  lx, ly = logM.shape
  K = np.full((lx + 1, ly + 1), -np.inf)
  K[0, 0] = 0.0
  for i in range(1, lx + 1):
    for j in range(1, ly + 1):
      a, b, c = K[i - 1, j], K[i, j - 1], K[i - 1, j - 1]
      m = max(a, b, c)
      K[i, j] = logM[i - 1, j - 1] + (
          m + np.log(np.exp(a - m) + np.exp(b - m) + np.exp(c - m)) if m > -np.inf else -np.inf)
  return K[lx, ly]


def global_align_kernel(X, Y=None, diag=False, kind='rbf', param=1.0):
  """FP64 ``GlobalAlignmentKernel(...)(X, Y, diag)`` (ksig/kernels.py:366-409
  with the log-space normalisation of :190-206; diag returns ones)."""
  Xs = as_seq_list(X)
  if diag:
    return np.ones((len(Xs),))
  Ys = Xs if Y is None else as_seq_list(Y)
  lk = np.array([[ga_log(static_gram(x, y, kind, param)) for y in Ys] for x in Xs])
  if Y is None:
    d = np.diagonal(lk)
    lk = lk - 0.5 * (d[:, None] + d[None, :])
  else:
    dx = np.array([ga_log(static_gram(x, x, kind, param)) for x in Xs])
    dy = np.array([ga_log(static_gram(y, y, kind, param)) for y in Ys])
    lk = lk - 0.5 * (dx[:, None] + dy[None, :])
  return np.exp(lk)
