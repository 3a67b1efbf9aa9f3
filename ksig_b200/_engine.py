"""Device-side calls into the C ABI on PyTorch CUDA tensors.

PyTorch only provides device memory and the current stream here; every
arithmetic step runs in ``libksig_b200.so``.
"""

import ctypes
import os

import numpy as np
import torch

from . import _lib as L


def _ptr(t):
  return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream():
  return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dtype_code(t):
  if t.dtype == torch.float64:
    return L.DTYPE_F64
  if t.dtype == torch.float32:
    return L.DTYPE_F32
  raise ValueError(f'unsupported dtype {t.dtype}; expected float32/float64')


def _workspace(nbytes, device):
  return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)


# Device-side checks (lengths outside [1, L], pair indices out of range,
# scratch geometry) never trap: the kernels record a status code in the
# first word of the call's workspace.  Every call folds that word into a
# per-device accumulator on the stream, without synchronising;
# check_device_status() reads and clears it at a point that synchronises
# anyway (the NumPy return of a kernel call) or when the caller asks.
_STATUS = {}


def _fold_status(ws):
  idx = ws.device.index if ws.device.index is not None else torch.cuda.current_device()
  acc = _STATUS.get(idx)
  if acc is None:
    acc = _STATUS[idx] = torch.zeros((1,), dtype=torch.int32, device=ws.device)
  torch.maximum(acc, ws[:4].view(torch.int32), out=acc)


def check_device_status():
  """Synchronises, then raises if a call since the last check recorded a
  device-side error: ValueError for invalid inputs (the reference's
  exception type), KsigError otherwise.  Clears the record."""
  for acc in _STATUS.values():
    code = int(acc.item())
    if code:
      acc.zero_()
      if code == L.ERR_INVALID:
        raise ValueError('device-side check failed: a sequence length is '
                         'outside [1, L] or a pair index is out of range')
      raise L.KsigError(code, f'device-side check failed (code {code})')


class Seqs:
  """A batch of sequences on the device: dense ``[n, L, d]`` plus lengths."""

  __slots__ = ('data', 'lengths', 'n', 'L', 'd')

  def __init__(self, data, lengths=None):
    if not data.is_cuda:
      raise ValueError('sequences must live on a CUDA device')
    self.data = data.contiguous()
    self.n, self.L, self.d = self.data.shape
    if lengths is not None:
      lengths = lengths.to(device=data.device, dtype=torch.int32).contiguous()
    self.lengths = lengths


def num_pairs(mode, nX, nY, n_list=0):
  return int(L.lib().ksig_num_pairs(mode, nX, nY, n_list))


def _static_args(kind, param):
  """(use_ex, float param, ctypes double[3]) for a static kernel given as
  one parameter (RBF, linear) or a parameter tuple (every kind)."""
  if isinstance(param, (tuple, list)):
    vals = [float(v) for v in param] + [0.0] * (3 - len(param))
    return True, vals[0], (ctypes.c_double * 3)(*vals[:3])
  if kind not in (L.STATIC_RBF, L.STATIC_LINEAR):
    raise ValueError('this static kernel needs its parameter tuple')
  return False, float(param), None


def sig_levels(X, Y, mode, n_levels, order, difference, kind, param,
               pair_list=None):
  """Per-level signature kernels ``[n_levels+1, P]`` (float64)."""
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  if Y is not None and Y.data.dtype != X.data.dtype:
    raise ValueError('X and Y must share a dtype')
  if Y is not None and Y.d != X.d:
    raise ValueError('X and Y must have the same number of features')
  n_list = 0 if pair_list is None else pair_list.shape[0]
  P = num_pairs(mode, X.n, Yv.n, n_list)
  out = torch.empty((n_levels + 1, max(P, 0)), dtype=torch.float64,
                    device=X.data.device)
  ws_bytes = lib.ksig_signature_kern_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, n_levels, order, int(difference), mode,
      n_list)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  ext, p0, pv = _static_args(kind, param)
  if ext:
    rc = lib.ksig_signature_kern_ex(
        _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
        _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, pv, n_levels,
        order, int(difference), mode, _ptr(pair_list), n_list, _ptr(out),
        _ptr(ws), ws_bytes, _stream())
  else:
    rc = lib.ksig_signature_kern(
        _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
        _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, p0, n_levels,
        order, int(difference), mode, _ptr(pair_list), n_list, _ptr(out),
        _ptr(ws), ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return out


def sig_levels_plain(X, Y, mode, n_levels, order, kind, param):
  """Per-level kernels from the plain one-pair-per-block baseline kernel."""
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  P = num_pairs(mode, X.n, Yv.n, 0)
  out = torch.empty((n_levels + 1, max(P, 0)), dtype=torch.float64,
                    device=X.data.device)
  ws_bytes = lib.ksig_signature_kern_plain_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, n_levels, order, mode, 0)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  rc = lib.ksig_signature_kern_plain(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
      _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, float(param), n_levels,
      order, mode, None, 0, _ptr(out), _ptr(ws), ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return out


def sig_levels_bwd(X, Y, mode, n_levels, order, kind, param, grad_levels,
                   dX=None, want_dparam=True, pair_list=None):
  """Row-side adjoint of :func:`sig_levels`.

  Accumulates into ``dX`` (``[nX, LX, d]``, X's dtype; allocated as zeros
  when None) and returns ``(dX, dparam)`` where dparam is a float64 device
  scalar (or None).
  """
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  n_list = 0 if pair_list is None else pair_list.shape[0]
  if dX is None:
    dX = torch.zeros_like(X.data)
  dpar = torch.zeros((1,), dtype=torch.float64, device=X.data.device) \
      if want_dparam else None
  gl = grad_levels.to(torch.float64).contiguous()
  ws_bytes = lib.ksig_signature_kern_bwd_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, n_levels, order, 1, mode, n_list)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  rc = lib.ksig_signature_kern_bwd(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
      _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, float(param), n_levels,
      order, 1, mode, _ptr(pair_list), n_list, _ptr(gl), _ptr(dX),
      _ptr(dpar), _ptr(ws), ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return dX, dpar


# Split-pass workspaces (up to tens of GB) handed back by the backward are
# kept per device for the next forwards: going through torch's cache
# instead, smaller tensors split the freed blocks and steps paid a new
# cudaMalloc of the whole workspace.  A released buffer carries an event
# recorded on the releasing stream after the backward's kernels; the stream
# that takes it waits on that event first, so a forward on another stream
# cannot overwrite records the adjoint is still reading.  The pool holds at
# most KSIG_REC_MB bytes per device.
_REC_POOL = {}
# Forwards that kept the split pass's records, and those that declined them
# (no compiled split pass, or records above rec_budget_bytes): a backward
# after a declined forward runs the one-launch adjoint.
REC_STATS = {'recorded': 0, 'declined': 0}


def _dev_index(device):
  return device.index if device.index is not None else torch.cuda.current_device()


def _rec_cap():
  return int(os.environ.get('KSIG_REC_MB', '65536')) << 20


def rec_budget_bytes(device):
  """Memory the split gradient pass may keep for its records:
  ``KSIG_REC_MB`` (default 65536), at most half of the available device
  memory: free memory plus what torch's cache holds unused (the largest
  pooled workspace counts as available too)."""
  free, _ = torch.cuda.mem_get_info(device)
  cached = torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
  pool = _REC_POOL.get(_dev_index(device), [])
  return min(_rec_cap(),
             (free + max(cached, 0)) // 2 + max((w.numel() for w in pool), default=0))


def _rec_take(nbytes, device):
  """The smallest pooled workspace of at least ``nbytes``, else a new one."""
  pool = _REC_POOL.setdefault(_dev_index(device), [])
  fit = [i for i, w in enumerate(pool) if w.numel() >= nbytes]
  if fit:
    ws = pool.pop(min(fit, key=lambda i: pool[i].numel()))
    ev = getattr(ws, '_ksig_released', None)
    if ev is not None:
      torch.cuda.current_stream(ws.device).wait_event(ev)
    return ws
  return _workspace(nbytes, device)


def rec_release(ws):
  """Hands a split-pass workspace back for reuse by the next forward."""
  pool = _REC_POOL.setdefault(_dev_index(ws.device), [])
  ev = torch.cuda.Event()
  ev.record(torch.cuda.current_stream(ws.device))
  ws._ksig_released = ev
  pool.append(ws)
  pool.sort(key=lambda w: -w.numel())
  while sum(w.numel() for w in pool) > _rec_cap():
    pool.pop()  # the smallest goes back to torch


def rec_pool_clear():
  """Drops the pooled split-pass workspaces (their memory returns to torch)."""
  _REC_POOL.clear()


def sig_levels_rec(X, Y, n_levels, order, kind, param, pair_list=None):
  """Forward of the split gradient pass (order 1): per-level kernels
  ``[n_levels+1, P]`` (float64) and the workspace holding the records of
  :func:`sig_levels_bwd_rec`, or None when the pass does not apply or its
  records exceed :func:`rec_budget_bytes`."""
  lib = L.lib()
  dt = _dtype_code(X.data)
  mode = L.PAIRS_FULL if pair_list is None else L.PAIRS_LIST
  n_list = 0 if pair_list is None else pair_list.shape[0]
  ws_bytes = lib.ksig_signature_kern_rec_workspace(
      X.n, X.L, Y.n, Y.L, X.d, dt, n_levels, order, 1, mode, n_list)
  if ws_bytes == 0 or ws_bytes > rec_budget_bytes(X.data.device):
    REC_STATS['declined'] += 1
    return None
  REC_STATS['recorded'] += 1
  P = num_pairs(mode, X.n, Y.n, n_list)
  out = torch.empty((n_levels + 1, max(P, 0)), dtype=torch.float64,
                    device=X.data.device)
  ws = _rec_take(ws_bytes, X.data.device)
  rc = lib.ksig_signature_kern_rec_fwd(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Y.data), _ptr(Y.lengths),
      Y.n, Y.L, X.d, dt, kind, float(param), n_levels, order, 1, mode,
      _ptr(pair_list), n_list, _ptr(out), _ptr(ws), ws.numel(), _stream())
  L.check(rc)
  _fold_status(ws)
  return out, ws


def sig_levels_bwd_rec(X, Y, n_levels, order, kind, param, grad_levels, ws,
                       dX=None, want_dparam=True, pair_list=None):
  """Adjoint pass of the split gradient pass: the records left in ``ws`` by
  :func:`sig_levels_rec` (same arguments) replace the forward recursion.
  Returns ``(dX, dparam)`` like :func:`sig_levels_bwd`."""
  lib = L.lib()
  dt = _dtype_code(X.data)
  mode = L.PAIRS_FULL if pair_list is None else L.PAIRS_LIST
  n_list = 0 if pair_list is None else pair_list.shape[0]
  if dX is None:
    dX = torch.zeros_like(X.data)
  dpar = torch.zeros((1,), dtype=torch.float64, device=X.data.device) \
      if want_dparam else None
  gl = grad_levels.to(torch.float64).contiguous()
  rc = lib.ksig_signature_kern_rec_bwd(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Y.data), _ptr(Y.lengths),
      Y.n, Y.L, X.d, dt, kind, float(param), n_levels, order, 1, mode,
      _ptr(pair_list), n_list, _ptr(gl), _ptr(dX), _ptr(dpar), _ptr(ws),
      ws.numel(), _stream())
  L.check(rc)
  _fold_status(ws)
  return dX, dpar


def sig_levels_bwd_plain(X, Y, mode, n_levels, order, kind, param, grad_levels,
                         dX=None, want_dparam=True):
  """Row-side adjoint from the plain one-pair-per-block baseline kernel
  (same contract as :func:`sig_levels_bwd`)."""
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  if dX is None:
    dX = torch.zeros_like(X.data)
  dpar = torch.zeros((1,), dtype=torch.float64, device=X.data.device) \
      if want_dparam else None
  gl = grad_levels.to(torch.float64).contiguous()
  ws_bytes = lib.ksig_signature_kern_plain_bwd_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, n_levels, order, mode, 0)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  rc = lib.ksig_signature_kern_plain_bwd(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
      _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, float(param), n_levels,
      order, mode, None, 0, _ptr(gl), _ptr(dX), _ptr(dpar), _ptr(ws),
      ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return dX, dpar


def ga_values(X, Y, mode, kind, param, pair_list=None):
  """Log global-alignment kernel per pair ``[P]`` (float64)."""
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  if Y is not None and Y.data.dtype != X.data.dtype:
    raise ValueError('X and Y must share a dtype')
  if Y is not None and Y.d != X.d:
    raise ValueError('X and Y must have the same number of features')
  n_list = 0 if pair_list is None else pair_list.shape[0]
  P = num_pairs(mode, X.n, Yv.n, n_list)
  out = torch.empty((max(P, 0),), dtype=torch.float64, device=X.data.device)
  ws_bytes = lib.ksig_global_align_kern_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, mode, n_list)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  rc = lib.ksig_global_align_kern(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
      _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, float(param), mode,
      _ptr(pair_list), n_list, _ptr(out), _ptr(ws), ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return out


def pde_values(X, Y, mode, dyadic_order, difference, kind, param,
               pair_list=None):
  """Signature-PDE kernel per pair ``[P]`` (float64)."""
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  if Y is not None and Y.data.dtype != X.data.dtype:
    raise ValueError('X and Y must share a dtype')
  if Y is not None and Y.d != X.d:
    raise ValueError('X and Y must have the same number of features')
  n_list = 0 if pair_list is None else pair_list.shape[0]
  P = num_pairs(mode, X.n, Yv.n, n_list)
  out = torch.empty((max(P, 0),), dtype=torch.float64, device=X.data.device)
  ws_bytes = lib.ksig_signature_kern_pde_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, dyadic_order, int(difference), mode,
      n_list)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  ext, p0, pv = _static_args(kind, param)
  if ext:
    rc = lib.ksig_signature_kern_pde_ex(
        _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
        _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, pv,
        dyadic_order, int(difference), mode, _ptr(pair_list), n_list,
        _ptr(out), _ptr(ws), ws_bytes, _stream())
  else:
    rc = lib.ksig_signature_kern_pde(
        _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
        _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, p0,
        dyadic_order, int(difference), mode, _ptr(pair_list), n_list,
        _ptr(out), _ptr(ws), ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return out


def normalize_levels(levels, mode, nX, nY, diagX, diagY, normalize,
                     out_dtype):
  """Normalisation / level mean (or level sum) -> ``[nX, nY]``."""
  n_lev = levels.shape[0]
  out = torch.empty((nX, nY), dtype=out_dtype, device=levels.device)
  code = L.DTYPE_F64 if out_dtype == torch.float64 else L.DTYPE_F32
  rc = L.lib().ksig_normalize_levels(
      _ptr(levels), n_lev, mode, nX, nY, _ptr(diagX), _ptr(diagY),
      int(normalize), _ptr(out), code, _stream())
  L.check(rc)
  return out


def to_numpy(t):
  return t.detach().cpu().numpy()


def np_dtype(t):
  return np.float64 if t.dtype == torch.float64 else np.float32


def pde_values_bwd(X, Y, mode, dyadic_order, kind, param, grad, dX=None,
                   want_dparam=True, pair_list=None):
  """Row-side adjoint of :func:`pde_values`; returns ``(dX, dparam)``."""
  lib = L.lib()
  Yv = X if Y is None else Y
  dt = _dtype_code(X.data)
  n_list = 0 if pair_list is None else pair_list.shape[0]
  if dX is None:
    dX = torch.zeros_like(X.data)
  dpar = torch.zeros((1,), dtype=torch.float64, device=X.data.device) \
      if want_dparam else None
  g = grad.to(torch.float64).contiguous()
  ws_bytes = lib.ksig_signature_kern_pde_bwd_workspace(
      X.n, X.L, Yv.n, Yv.L, X.d, dt, dyadic_order, 1, mode, n_list)
  if ws_bytes == 0:
    L.check(L.ERR_UNSUPPORTED if 'no compiled' in L.last_error()
            else L.ERR_INVALID)
  ws = _workspace(ws_bytes, X.data.device)
  rc = lib.ksig_signature_kern_pde_bwd(
      _ptr(X.data), _ptr(X.lengths), X.n, X.L, _ptr(Yv.data),
      _ptr(Yv.lengths), Yv.n, Yv.L, X.d, dt, kind, float(param),
      dyadic_order, 1, mode, _ptr(pair_list), n_list, _ptr(g), _ptr(dX),
      _ptr(dpar), _ptr(ws), ws_bytes, _stream())
  L.check(rc)
  _fold_status(ws)
  return dX, dpar
