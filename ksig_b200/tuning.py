"""Autotuner for the sweep tile width (no reference counterpart).

The sweep kernels are compiled for several column counts per lane C (a
strip is 32*C - 1 cells wide).  The built-in choice takes the narrowest
strip that covers the longest column sequence; the best width also depends
on the length mix of a ragged batch, on d, the level count and the order.
:func:`autotune` times the compiled widths on the caller's own inputs and
keeps the fastest for the kernel family (process-wide, through
``ksig_tune_set_cols``); results are cached per workload key.
"""

import torch

from . import _lib as L
from .kernels import SignaturePDEKernel

OP_DP_FWD, OP_PDE_FWD, OP_DP_BWD, OP_PDE_BWD = 0, 1, 2, 3
WIDTHS = {OP_DP_FWD: (2, 4, 7), OP_PDE_FWD: (2, 4, 8),
          OP_DP_BWD: (2, 4, 7), OP_PDE_BWD: (2, 4, 8)}

_cache = {}


def _shape_key(X):
  from .kernels import Ragged
  if X is None:
    return None
  if isinstance(X, Ragged):
    return ('ragged', tuple(X.data.shape), str(X.data.dtype))
  if isinstance(X, torch.Tensor):
    return ('dense', tuple(X.shape), str(X.dtype))
  return ('list', len(X))


def _time(fn, reps):
  fn()
  torch.cuda.synchronize()
  best = None
  for _ in range(reps):
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    b.synchronize()
    t = a.elapsed_time(b)
    best = t if best is None else min(best, t)
  return best


def set_cols(op, cols):
  L.check(L.lib().ksig_tune_set_cols(op, int(cols)))


def get_cols(op):
  return int(L.lib().ksig_tune_get_cols(op))


def autotune(kernel, X, Y=None, backward=False, reps=3):
  """Picks the fastest compiled tile width for ``kernel(X, Y)`` (and, with
  ``backward``, for its adjoint on ``sum(kernel(X, Y))``).

  Returns ``{op: (cols, ms)}``; the choice stays in effect for later calls
  of that kernel family until :func:`reset`.
  """
  pde = isinstance(kernel, SignaturePDEKernel)
  fwd_op = OP_PDE_FWD if pde else OP_DP_FWD
  key = (type(kernel).__name__, getattr(kernel, 'n_levels', None),
         getattr(kernel, 'order', None), getattr(kernel, 'dyadic_order', None),
         _shape_key(X), _shape_key(Y), backward)
  if key in _cache:
    for op, (c, _) in _cache[key].items():
      set_cols(op, c)
    return _cache[key]
  result = {}

  def fwd():
    kernel(X, Y, return_on_gpu=True)

  times = {}
  for c in WIDTHS[fwd_op]:
    set_cols(fwd_op, c)
    try:
      times[c] = _time(fwd, reps)
    except (ValueError, NotImplementedError, RuntimeError):
      continue
  if times:
    c = min(times, key=times.get)
    set_cols(fwd_op, c)
    result[fwd_op] = (c, times[c])
  if backward:
    from .kernels import Ragged
    bwd_op = OP_PDE_BWD if pde else OP_DP_BWD
    if isinstance(X, Ragged):
      Xg = Ragged(X.data.detach().clone().requires_grad_(True), X.lengths)
      grad_of = Xg.data
    else:
      Xg = X.detach().clone().requires_grad_(True)
      grad_of = Xg

    def fb():
      grad_of.grad = None
      kernel(Xg, Y, return_on_gpu=True).sum().backward()

    times = {}
    for c in WIDTHS[bwd_op]:
      set_cols(bwd_op, c)
      try:
        times[c] = _time(fb, reps)
      except (ValueError, NotImplementedError, RuntimeError):
        continue
    if times:
      c = min(times, key=times.get)
      set_cols(bwd_op, c)
      result[bwd_op] = (c, times[c])
  _cache[key] = result
  return result


def reset():
  """Back to the built-in widths for every kernel family."""
  for op in WIDTHS:
    set_cols(op, 0)
