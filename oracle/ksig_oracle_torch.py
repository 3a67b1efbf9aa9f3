"""FP64 PyTorch restatement of the oracle recursions, for gradient checks.

Test infrastructure (the checker, never the product).  The same algorithms
as ``ksig_oracle.py`` (ksig/algorithms.py:47-140 for the DP kernel,
ksig/algorithms.py:344-399 for the Goursat PDE, ksig/static/kernels.py:248-260
and :145-155 for the static kernels, ksig/kernels.py:180-214 for the
normalisation) written with differentiable torch ops on CPU float64, so that
autograd provides reference gradients with respect to the inputs and the
static-kernel parameter.  The reference itself has no gradients, so these are
pinned by central finite differences instead (tests/test_oracle_grad.py).
"""

import torch

EPS = 1e-12


def static_gram(X, Y, kind='rbf', param=1.0):
  xy = torch.einsum('...ij,...kj->...ik', X, Y)
  if kind == 'rbf':
    xn = (X * X).sum(-1)
    yn = (Y * Y).sum(-1)
    d2 = xn[..., :, None] + yn[..., None, :] - 2 * xy
    if isinstance(param, torch.Tensor):
      denom = torch.clamp(2 * param ** 2, min=EPS)
    else:
      denom = max(2 * param ** 2, EPS)
    return torch.exp(-d2 / denom)
  return param * xy


def _excl(M, axes):
  """Exclusive cumsum over ``axes`` (ksig/utils.py:63-90)."""
  for a in axes:
    M = torch.cumsum(M, dim=a)
    pad = [0, 0] * (M.ndim - 1 - (a % M.ndim)) + [1, 0]
    sl = [slice(None)] * M.ndim
    sl[a] = slice(0, -1)
    M = torch.nn.functional.pad(M[tuple(sl)], pad)
  return M


def sig_levels(Z, n_levels, order=1):
  """Per-level kernels ``[n_levels+1, ...]`` (Alg. 3 / Alg. 6)."""
  order = n_levels if order <= 0 or order >= n_levels else order
  K = [torch.ones(Z.shape[:-2], dtype=Z.dtype), Z.sum((-2, -1))]
  if order == 1:
    R = Z
    for _ in range(1, n_levels):
      R = Z * _excl(R, (-2, -1))
      K.append(R.sum((-2, -1)))
    return torch.stack(K, 0)
  R = {(0, 0): Z}
  dprev = 1
  for i in range(1, n_levels):
    d = min(i + 1, order)
    Rn = {}
    A = sum(R[(a, b)] for a in range(dprev) for b in range(dprev))
    Rn[(0, 0)] = Z * _excl(A, (-2, -1))
    for r in range(1, d):
      V = sum(R[(a, r - 1)] for a in range(dprev))
      U = sum(R[(r - 1, b)] for b in range(dprev))
      Rn[(0, r)] = Z * _excl(V, (-2,)) / (r + 1)
      Rn[(r, 0)] = Z * _excl(U, (-1,)) / (r + 1)
      for s in range(1, d):
        Rn[(r, s)] = Z * R[(r - 1, s - 1)] / ((r + 1) * (s + 1))
    R = Rn
    dprev = d
    K.append(sum(v.sum((-2, -1)) for v in R.values()))
  return torch.stack(K, 0)


def sig_pde(Z, dyadic_order=0):
  f = 2 ** dyadic_order
  if f > 1:
    Z = torch.repeat_interleave(torch.repeat_interleave(Z, f, -2), f, -1) / (f * f)
  lx, ly = Z.shape[-2:]
  lead = Z.shape[:-2]
  A = 1 + 0.5 * Z + Z * Z / 12
  B = 1 - Z * Z / 12
  one = torch.ones(lead, dtype=Z.dtype)
  prev = [one] * (ly + 1)          # K[i, :]
  for i in range(lx):
    cur = [one]
    for j in range(ly):
      cur.append((prev[j + 1] + cur[j]) * A[..., i, j] - prev[j] * B[..., i, j])
    prev = cur
  return prev[ly]


def _diff2(M):
  return M[..., 1:, 1:] - M[..., 1:, :-1] - M[..., :-1, 1:] + M[..., :-1, :-1]


def pair_value(x, y, kind, param, fn, difference=True):
  M = static_gram(x, y, kind, param)
  return fn(_diff2(M) if difference else M)


def gram(Xs, Ys, kind, param, fn, difference=True):
  """Per-pair values ``[..., nX, nY]`` for lists of ``[L_i, d]`` tensors."""
  rows = []
  for x in Xs:
    rows.append(torch.stack([pair_value(x, y, kind, param, fn, difference)
                             for y in Ys], -1))
  return torch.stack(rows, -2)


def signature_kernel(Xs, Ys=None, n_levels=5, order=1, normalize=True,
                     kind='rbf', param=1.0, difference=True):
  fn = lambda Z: sig_levels(Z, n_levels, order)  # noqa: E731
  return _front(Xs, Ys, normalize, kind, param, fn, difference)


def signature_pde_kernel(Xs, Ys=None, normalize=True, kind='rbf', param=1.0,
                         dyadic_order=0, difference=True):
  fn = lambda Z: sig_pde(Z, dyadic_order)  # noqa: E731
  return _front(Xs, Ys, normalize, kind, param, fn, difference)


def _front(Xs, Ys, normalize, kind, param, fn, difference):
  sym = Ys is None
  Ys = Xs if sym else Ys
  K = gram(Xs, Ys, kind, param, fn, difference)
  if not normalize:
    return K.sum(0) if K.ndim == 3 else K
  if sym:
    Kx = torch.diagonal(K, dim1=-2, dim2=-1)
    Ky = Kx
  else:
    Kx = torch.stack([pair_value(x, x, kind, param, fn, difference) for x in Xs], -1)
    Ky = torch.stack([pair_value(y, y, kind, param, fn, difference) for y in Ys], -1)
  sx = torch.clamp(torch.sqrt(torch.clamp(Kx, min=EPS)), min=EPS)
  sy = torch.clamp(torch.sqrt(torch.clamp(Ky, min=EPS)), min=EPS)
  K = K / (sx[..., :, None] * sy[..., None, :])
  return K.mean(0) if K.ndim == 3 else K
