"""torch.autograd.Function around the signature-kernel forward and adjoint.

Forward: level kernels from the fused CUDA sweep, then the normalisation of
ksig/kernels.py:190-214.  Backward: the chain rule through the
normalisation is a few O(n_levels * nX * nY) FP64 tensor ops; the adjoint of
the level kernels themselves (the expensive part) runs in the CUDA adjoint
sweep, which differentiates the row sequence of each pair.  Column-side
gradients come from a second sweep with the roles of X and Y swapped; for
K(X) one sweep over all ordered pairs with symmetrised weights covers both
sides (diagonal pairs weighted twice).
"""

import torch

from . import _engine as E
from . import _lib as L
from .utils import _EPS


def _upper_index(n, device):
  a, b = torch.triu_indices(n, n, device=device)
  return a, b


def _full_from_upper(lev, n):
  """[n_lev, n(n+1)/2] row-major upper triangle -> symmetric [n_lev, n, n]."""
  a, b = _upper_index(n, lev.device)
  out = torch.empty((lev.shape[0], n, n), dtype=lev.dtype, device=lev.device)
  out[:, a, b] = lev
  out[:, b, a] = lev
  return out


def _norm_scale(Kd):
  """max(robust_sqrt(Kd), eps) and its derivative w.r.t. Kd."""
  r = torch.sqrt(torch.clamp(Kd, min=_EPS))
  s = torch.clamp(r, min=_EPS)
  ds = torch.where((Kd > _EPS) & (r > _EPS), 0.5 / r, torch.zeros_like(r))
  return s, ds


class SigKernelFn(torch.autograd.Function):
  """K = normalised (or summed) signature Gram; differentiable in X, Y and
  the static-kernel parameter."""

  @staticmethod
  def forward(ctx, Xt, Yt, pt, spec):
    # spec: dict(n_levels, order, normalize, kind, param, Xs, Ys, levels_fn)
    Xs, Ys = spec['Xs'], spec['Ys']
    lev_fn = spec['levels_fn']
    sym = Ys is None
    out_dtype = Xs.data.dtype
    split = spec.get('rec_fn')
    use_split = split is not None and (Xt is not None or pt is not None)
    if sym:
      # The backward differentiates all ordered pairs; with the split pass
      # the forward records them all and keeps the upper triangle.
      rec = split[0](Xs, Xs) if use_split else None
      if rec is not None:
        levf, ctx.rec_ws = rec
        a, b = _upper_index(Xs.n, levf.device)
        lev = levf[:, a * Xs.n + b].contiguous()
      else:
        lev = lev_fn(Xs, None, L.PAIRS_UPPER)
      K = E.normalize_levels(lev, L.PAIRS_UPPER, Xs.n, Xs.n, None, None,
                             spec['normalize'], out_dtype)
      dx = dy = None
    else:
      # Split gradient pass: the forward keeps the adjoint's records, the
      # backward replays them (see SignatureKernel._split_pass).
      rec = split[0](Xs, Ys) if use_split else None
      if rec is not None:
        lev, ctx.rec_ws = rec
      else:
        lev = lev_fn(Xs, Ys, L.PAIRS_FULL)
      dx = dy = None
      if spec['normalize']:
        dx = lev_fn(Xs, None, L.PAIRS_DIAG)
        dy = lev_fn(Ys, None, L.PAIRS_DIAG)
      K = E.normalize_levels(lev, L.PAIRS_FULL, Xs.n, Ys.n, dx, dy,
                             spec['normalize'], out_dtype)
    if not hasattr(ctx, 'rec_ws'):
      ctx.rec_ws = None
    ctx.spec = spec
    ctx.sym = sym
    ctx.saved = (lev, dx, dy)
    ctx.x_meta = (Xt.shape, Xt.dtype, Xt.device) if Xt is not None else None
    ctx.y_meta = (Yt.shape, Yt.dtype, Yt.device) if Yt is not None else None
    return K

  @staticmethod
  def backward(ctx, G):
    spec = ctx.spec
    lev, dx, dy = ctx.saved
    Xs, Ys = spec['Xs'], spec['Ys']
    G = G.to(torch.float64)
    n_lev = lev.shape[0]
    nX = Xs.n
    nY = nX if ctx.sym else Ys.n
    Klf = _full_from_upper(lev, nX) if ctx.sym else lev.view(n_lev, nX, nY)
    if spec['normalize']:
      Kx = torch.diagonal(Klf, dim1=1, dim2=2) if ctx.sym else dx
      Ky = Kx if ctx.sym else dy
      sx, dsx = _norm_scale(Kx)
      sy, dsy = _norm_scale(Ky)
      denom = sx[:, :, None] * sy[:, None, :]
      gK = G[None] / (n_lev * denom)                       # dL/dK_l
      t = gK * Klf                                        # G K_l / (n s s)
      gKx = -(t.sum(2) / sx) * dsx                          # dL/dKx_l
      gKy = -(t.sum(1) / sy) * dsy                          # dL/dKy_l
    else:
      gK = G[None].expand(n_lev, nX, nY).clone()
      gKx = gKy = None
    if spec.get('const_level0', True):
      gK[0] = 0.0  # DP level 0 is the constant 1
    want_x = ctx.needs_input_grad[0]
    want_y = ctx.needs_input_grad[1]
    want_p = ctx.needs_input_grad[2]
    kind, param = spec['kind'], spec['param']
    bwd = spec['bwd_fn']
    dX = dY = dP = None
    dpar_total = torch.zeros((1,), dtype=torch.float64, device=G.device)
    if ctx.sym:
      if gKx is not None:
        idx = torch.arange(nX, device=G.device)
        gK[:, idx, idx] += gKx + gKy
      W = gK + gK.transpose(1, 2)  # diagonal counted twice: both sides
      if want_x or want_p:
        if ctx.rec_ws is not None:
          dXd, dp = spec['rec_fn'][1](Xs, Xs, W.reshape(n_lev, -1), want_p,
                                      ctx.rec_ws)
        else:
          dXd, dp = bwd(Xs, Xs, L.PAIRS_FULL, W.reshape(n_lev, -1), want_p)
        dX = dXd if want_x else None
        if dp is not None:
          dpar_total += 0.5 * dp
    else:
      if want_x or want_p:
        if ctx.rec_ws is not None:
          dXd, dp = spec['rec_fn'][1](Xs, Ys, gK.reshape(n_lev, -1), want_p,
                                      ctx.rec_ws)
        else:
          dXd, dp = bwd(Xs, Ys, L.PAIRS_FULL, gK.reshape(n_lev, -1), want_p)
        dX = dXd
        if dp is not None:
          dpar_total += dp
      if want_y:
        dYd, _ = bwd(Ys, Xs, L.PAIRS_FULL,
                     gK.transpose(1, 2).reshape(n_lev, -1), False)
        dY = dYd
      if gKx is not None:
        if want_x or want_p:
          dXd2, dp = bwd(Xs, None, L.PAIRS_DIAG, 2.0 * gKx, want_p)
          dX = dXd2 if dX is None else dX + dXd2
          if dp is not None:
            dpar_total += 0.5 * dp
        if want_y or want_p:
          dYd2, dp = bwd(Ys, None, L.PAIRS_DIAG, 2.0 * gKy, want_p)
          if want_y:
            dY = dYd2 if dY is None else dY + dYd2
          if dp is not None:
            dpar_total += 0.5 * dp
    if ctx.rec_ws is not None:  # the records are used once
      E.rec_release(ctx.rec_ws)
      ctx.rec_ws = None
    gx = gy = None
    if want_x and dX is not None and ctx.x_meta is not None:
      shape, dtype, device = ctx.x_meta
      gx = dX.to(device=device, dtype=dtype).reshape(shape)
    if want_y and dY is not None and ctx.y_meta is not None:
      shape, dtype, device = ctx.y_meta
      gy = dY.to(device=device, dtype=dtype).reshape(shape)
    if want_p:
      dP = dpar_total.reshape(()).to(spec['param_dtype'])
      dP = dP.to(spec['param_device'])
    return gx, gy, dP, None
