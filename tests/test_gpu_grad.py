"""Gradients of the CUDA adjoint against autograd through the FP64 torch
oracle (itself pinned to central finite differences in
tests/test_oracle_grad.py).

Bar (normwise, stated here on purpose): max_i |g_i - r_i| / max_i |r_i| <=
1e-4 for FP32 inputs and 1e-8 for FP64 inputs, over each gradient tensor;
outputs are checked per entry.  The per-coordinate bar (|g_i - r_i| <= 1e-4
max(|r_i|, 1e-2 max |r|)) is applied at the large shapes in
tests/test_gpu_config5.py and tests/test_gpu_coverage.py."""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle_torch as OT

pytestmark = pytest.mark.gpu


def _walks(rng, n, L, d, scale=0.3):
  return np.cumsum(rng.standard_normal((n, L, d)) * scale, axis=1)


def _relerr(a, b):
  a = a.detach().cpu().double().numpy()
  b = b.detach().cpu().double().numpy()
  return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _run(kern_factory, oracle_fn, X, Y, bw, dt, tol, sym=False):
  import ksig_b200 as K
  w_rng = np.random.default_rng(123)
  # ours
  Xt = torch.tensor(X, dtype=dt, device='cuda', requires_grad=True)
  Yt = None if sym else torch.tensor(Y, dtype=dt, device='cuda', requires_grad=True)
  bt = torch.tensor(bw, dtype=torch.float64, requires_grad=True)
  kern = kern_factory(K, bt)
  out = kern(Xt) if sym else kern(Xt, Yt)
  W = torch.tensor(w_rng.standard_normal(tuple(out.shape)), device='cuda',
                   dtype=out.dtype)
  (out * W).sum().backward()
  # oracle on the same (rounded) inputs
  Xo = [torch.tensor(x, dtype=torch.float64, requires_grad=True)
        for x in Xt.detach().double().cpu().numpy()]
  Yo = None if sym else [torch.tensor(y, dtype=torch.float64, requires_grad=True)
                         for y in Yt.detach().double().cpu().numpy()]
  bo = torch.tensor(bw, dtype=torch.float64, requires_grad=True)
  ref = oracle_fn(Xo, Yo, bo)
  assert _relerr(out, ref) < tol
  (ref * W.double().cpu()).sum().backward()
  gX = torch.stack([x.grad for x in Xo])
  assert _relerr(Xt.grad, gX) < tol, ('dX', _relerr(Xt.grad, gX))
  if not sym:
    gY = torch.stack([y.grad for y in Yo])
    assert _relerr(Yt.grad, gY) < tol, ('dY', _relerr(Yt.grad, gY))
  assert abs(bt.grad.item() - bo.grad.item()) <= tol * max(1.0, abs(bo.grad.item())), \
      ('dbw', bt.grad.item(), bo.grad.item())


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-8), (torch.float32, 1e-4)])
@pytest.mark.parametrize('normalize', [True, False])
@pytest.mark.parametrize('order,n_levels', [(1, 4), (2, 4), (3, 5)])
def test_dp_grad_rect(dt, tol, normalize, order, n_levels):
  rng = np.random.default_rng(order * 7 + n_levels)
  X = _walks(rng, 3, 23, 3)
  Y = _walks(rng, 2, 17, 3)
  _run(lambda K, b: K.SignatureKernel(n_levels=n_levels, order=order,
                                      normalize=normalize,
                                      static_kernel=K.RBFKernel(b)),
       lambda x, y, b: OT.signature_kernel(x, y, n_levels=n_levels,
                                           order=order, normalize=normalize,
                                           param=b),
       X, Y, 0.8, dt, tol)


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-8), (torch.float32, 1e-4)])
@pytest.mark.parametrize('normalize', [True, False])
def test_dp_grad_sym(dt, tol, normalize):
  rng = np.random.default_rng(5)
  X = _walks(rng, 4, 19, 2)
  _run(lambda K, b: K.SignatureKernel(n_levels=5, order=1, normalize=normalize,
                                      static_kernel=K.RBFKernel(b)),
       lambda x, y, b: OT.signature_kernel(x, None, n_levels=5, order=1,
                                           normalize=normalize, param=b),
       X, None, 0.7, dt, tol, sym=True)


def test_dp_grad_linear_fp64():
  rng = np.random.default_rng(8)
  X = _walks(rng, 2, 15, 3)
  Y = _walks(rng, 3, 12, 3)
  _run(lambda K, b: K.SignatureKernel(n_levels=4, order=2, normalize=True,
                                      static_kernel=K.LinearKernel(b)),
       lambda x, y, b: OT.signature_kernel(x, y, n_levels=4, order=2,
                                           normalize=True, kind='linear',
                                           param=b),
       X, Y, 0.6, torch.float64, 1e-8)


@pytest.mark.parametrize('L', [140, 300])
def test_dp_grad_multi_strip_fp64(L):
  rng = np.random.default_rng(L)
  X = _walks(rng, 2, L, 2, scale=0.1)
  Y = _walks(rng, 1, L - 9, 2, scale=0.1)
  _run(lambda K, b: K.SignatureKernel(n_levels=3, order=2, normalize=True,
                                      static_kernel=K.RBFKernel(b)),
       lambda x, y, b: OT.signature_kernel(x, y, n_levels=3, order=2,
                                           normalize=True, param=b),
       X, Y, 0.9, torch.float64, 1e-8)


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-8), (torch.float32, 1e-4)])
@pytest.mark.parametrize('dyadic', [0, 1, 2])
@pytest.mark.parametrize('normalize', [False, True])
def test_pde_grad_rect(dt, tol, dyadic, normalize):
  rng = np.random.default_rng(20 + dyadic)
  X = _walks(rng, 2, 9, 3)
  Y = _walks(rng, 2, 7, 3)
  _run(lambda K, b: K.SignaturePDEKernel(normalize=normalize, dyadic_order=dyadic,
                                         static_kernel=K.RBFKernel(b)),
       lambda x, y, b: OT.signature_pde_kernel(x, y, normalize=normalize,
                                               dyadic_order=dyadic, param=b),
       X, Y, 0.9, dt, tol)


def test_pde_grad_sym_fp64():
  rng = np.random.default_rng(31)
  X = _walks(rng, 3, 8, 2)
  _run(lambda K, b: K.SignaturePDEKernel(normalize=True, dyadic_order=1,
                                         static_kernel=K.RBFKernel(b)),
       lambda x, y, b: OT.signature_pde_kernel(x, None, normalize=True,
                                               dyadic_order=1, param=b),
       X, None, 0.8, torch.float64, 1e-8, sym=True)


def test_pde_grad_linear_multistrip_fp64():
  """Column sequence longer than one strip of the adjoint (C = 2 lanes)."""
  import os
  os.environ['KSIG_BWD_COLS'] = '2'
  try:
    rng = np.random.default_rng(32)
    X = _walks(rng, 1, 12, 2, scale=0.1)
    Y = _walks(rng, 1, 80, 2, scale=0.05)
    _run(lambda K, b: K.SignaturePDEKernel(normalize=False, dyadic_order=0,
                                           static_kernel=K.LinearKernel(b)),
         lambda x, y, b: OT.signature_pde_kernel(x, y, normalize=False,
                                                 kind='linear', param=b),
         X, Y, 0.7, torch.float64, 1e-8)
  finally:
    del os.environ['KSIG_BWD_COLS']


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-9), (torch.float32, 1e-4)])
@pytest.mark.parametrize('order,n_levels,kind', [(1, 5, 0), (2, 4, 0), (3, 4, 1)])
def test_plain_bwd_baseline_matches_fused(dt, tol, order, n_levels, kind):
  """The plain one-pair-per-block adjoint gives the fused adjoint's dX and
  dparam on ragged inputs (the fused one is pinned to the oracle above)."""
  from ksig_b200 import _engine as E
  rng = np.random.default_rng(40 + order)
  X = torch.tensor(_walks(rng, 3, 21, 3), dtype=dt, device='cuda')
  Y = torch.tensor(_walks(rng, 4, 26, 3), dtype=dt, device='cuda')
  lx = torch.tensor([21, 9, 15], dtype=torch.int32, device='cuda')
  ly = torch.tensor([26, 4, 19, 11], dtype=torch.int32, device='cuda')
  Xs, Ys = E.Seqs(X, lx), E.Seqs(Y, ly)
  gl = torch.tensor(rng.standard_normal((n_levels + 1, 12)), device='cuda')
  param = 0.9 if kind == 0 else 0.7
  dXf, dpf = E.sig_levels_bwd(Xs, Ys, 0, n_levels, order, kind, param, gl)
  dXp, dpp = E.sig_levels_bwd_plain(Xs, Ys, 0, n_levels, order, kind, param, gl)
  assert _relerr(dXp, dXf) < tol
  assert abs(dpp.item() - dpf.item()) <= tol * max(1.0, abs(dpf.item()))


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-8), (torch.float32, 1e-4)])
def test_dp_grad_deep_truncation(dt, tol):
  rng = np.random.default_rng(98)
  X = _walks(rng, 2, 14, 2)
  Y = _walks(rng, 2, 11, 2)
  _run(lambda K, b: K.SignatureKernel(n_levels=10, order=1, normalize=True,
                                      static_kernel=K.RBFKernel(b)),
       lambda x, y, b: OT.signature_kernel(x, y, n_levels=10, order=1,
                                           normalize=True, param=b),
       X, Y, 0.9, dt, tol)


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-10), (torch.float32, 2e-6)])
@pytest.mark.parametrize('L,ragged', [(40, False), (260, False), (150, True)])
@pytest.mark.parametrize('kind', ['rbf', 'linear'])
def test_split_gradient_pass_matches_one_launch(dt, tol, L, ragged, kind):
  """ksig_signature_kern_rec_fwd / _rec_bwd (forward pass with per-pair
  records, then the adjoint pass alone) against ksig_signature_kern and
  ksig_signature_kern_bwd: levels, dX and dparam, single- and multi-strip
  (260 columns), ragged lengths."""
  from ksig_b200 import _engine as E, _lib as Lb
  rng = np.random.default_rng(L + 7 * ragged)
  X = torch.tensor(_walks(rng, 3, L, 4), dtype=dt, device='cuda')
  Y = torch.tensor(_walks(rng, 4, L + 13, 4), dtype=dt, device='cuda')
  lx = ly = None
  if ragged:
    lx = torch.tensor([L, L // 2, 7], dtype=torch.int32, device='cuda')
    ly = torch.tensor([L + 13, 3, L // 3, 1], dtype=torch.int32, device='cuda')
  Xs, Ys = E.Seqs(X, lx), E.Seqs(Y, ly)
  k = Lb.STATIC_RBF if kind == 'rbf' else Lb.STATIC_LINEAR
  par = 0.9 if kind == 'rbf' else 0.7
  m = 5
  ref = E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, m, 1, True, k, par)
  out = E.sig_levels_rec(Xs, Ys, m, 1, k, par)
  assert out is not None
  lev, ws = out
  assert _relerr(lev, ref) < tol
  gl = torch.tensor(np.random.default_rng(3).standard_normal(tuple(ref.shape)),
                    device='cuda')
  dX0, dp0 = E.sig_levels_bwd(Xs, Ys, Lb.PAIRS_FULL, m, 1, k, par, gl)
  dX1, dp1 = E.sig_levels_bwd_rec(Xs, Ys, m, 1, k, par, gl, ws)
  assert _relerr(dX1, dX0) < tol
  assert abs(dp1.item() - dp0.item()) <= tol * max(1.0, abs(dp0.item()))


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-10), (torch.float32, 2e-6)])
@pytest.mark.parametrize('sym', [False, True])
def test_split_gradient_pass_through_autograd(dt, tol, sym, monkeypatch):
  """K(X, Y) and K(X) gradients with the split pass (default) and without
  it (KSIG_REC_MB=0), normalised, the inputs and the bandwidth requiring
  grad."""
  import ksig_b200 as K
  rng = np.random.default_rng(11)
  X = _walks(rng, 3, 70, 3)
  Y = _walks(rng, 2, 90, 3)

  def run():
    Xt = torch.tensor(X, dtype=dt, device='cuda', requires_grad=True)
    Yt = torch.tensor(Y, dtype=dt, device='cuda', requires_grad=True)
    bt = torch.tensor(0.8, dtype=torch.float64, requires_grad=True)
    kern = K.SignatureKernel(n_levels=4, order=1, static_kernel=K.RBFKernel(bt))
    out = kern(Xt) if sym else kern(Xt, Yt)
    W = torch.tensor(np.random.default_rng(5).standard_normal(tuple(out.shape)),
                     device='cuda', dtype=out.dtype)
    (out * W).sum().backward()
    gy = torch.zeros(1) if sym else Yt.grad
    return out.detach(), Xt.grad, gy, bt.grad
  a = run()
  monkeypatch.setenv('KSIG_REC_MB', '0')
  b = run()
  for u, v in zip(a, b):
    assert _relerr(u, v) < tol


def test_split_pass_workspace_reused():
  """The backward hands the split pass's workspace back and the next
  forward takes the same buffer (no new allocation per step)."""
  import ksig_b200 as K
  from ksig_b200 import _engine as E
  rng = np.random.default_rng(12)
  X = torch.tensor(_walks(rng, 3, 60, 3), dtype=torch.float32, device='cuda',
                   requires_grad=True)
  Y = torch.tensor(_walks(rng, 2, 50, 3), dtype=torch.float32, device='cuda')
  kern = K.SignatureKernel(n_levels=4, order=1, static_kernel=K.RBFKernel(0.8))
  E.rec_pool_clear()
  ptrs = []
  for _ in range(3):
    kern(X, Y).sum().backward()
    pool = E._REC_POOL[torch.cuda.current_device()]
    assert len(pool) == 1
    ptrs.append(pool[0].data_ptr())
  assert ptrs[0] == ptrs[1] == ptrs[2]
  E.rec_pool_clear()


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-12), (torch.float32, 2e-6)])
@pytest.mark.parametrize('order,m', [(1, 5), (2, 4)])
def test_dp_adjoint_strip_checkpointing(dt, tol, order, m, monkeypatch):
  """Strip checkpointing (one strip of records, the others recomputed from
  their checkpoints in the adjoint pass) gives the same dX and dparam as
  keeping every strip's records, on ragged multi-strip pairs, in a smaller
  workspace."""
  from ksig_b200 import _engine as E, _lib as Lb
  rng = np.random.default_rng(60 + order)
  X = torch.tensor(_walks(rng, 3, 90, 3, 0.1), dtype=dt, device='cuda')
  Y = torch.tensor(_walks(rng, 4, 700, 3, 0.1), dtype=dt, device='cuda')
  lx = torch.tensor([90, 41, 7], dtype=torch.int32, device='cuda')
  ly = torch.tensor([700, 3, 333, 512], dtype=torch.int32, device='cuda')
  Xs, Ys = E.Seqs(X, lx), E.Seqs(Y, ly)
  gl = torch.tensor(np.random.default_rng(4).standard_normal((m + 1, 12)), device='cuda')
  lib = Lb.lib()
  dt_code = Lb.DTYPE_F64 if dt == torch.float64 else Lb.DTYPE_F32
  sizes = {}
  out = {}
  for ck in ('0', '1'):
    monkeypatch.setenv('KSIG_DP_BWD_CKPT', ck)
    sizes[ck] = lib.ksig_signature_kern_bwd_workspace(3, 90, 4, 700, 3, dt_code, m, order, 1,
                                                      Lb.PAIRS_FULL, 0)
    out[ck] = E.sig_levels_bwd(Xs, Ys, Lb.PAIRS_FULL, m, order, Lb.STATIC_RBF, 0.9, gl)
  assert sizes['1'] < sizes['0']
  assert _relerr(out['1'][0], out['0'][0]) < tol
  assert abs(out['1'][1].item() - out['0'][1].item()) <= tol * max(1.0, abs(out['0'][1].item()))
  # and against autograd through the FP64 oracle
  Xo = [torch.tensor(x[:int(n)].double().cpu().numpy(), requires_grad=True) for x, n in zip(X, lx)]
  Yo = [torch.tensor(y[:int(n)].double().cpu().numpy()) for y, n in zip(Y, ly)]
  ref = OT.gram(Xo, Yo, 'rbf', 0.9, lambda Z: OT.sig_levels(Z, m, order))
  (ref * gl.double().cpu().reshape(m + 1, 3, 4)).sum().backward()
  g = out['1'][0].double().cpu()
  for i, (x, n) in enumerate(zip(Xo, lx)):
    gi = g[i, :int(n)]
    assert float((gi - x.grad).abs().max() / x.grad.abs().max()) < (1e-8 if dt == torch.float64 else 1e-4)
