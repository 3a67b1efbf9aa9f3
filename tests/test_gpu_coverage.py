"""Shapes beyond the register-Gram tiles, against the FP64 oracle.

- More channels than the widest register tile (d > 32): the forward runs the
  Gram-input sweep (a precomputed Gram slot per task, in chunks of tasks);
  the DP adjoint runs the plain one-pair-per-block kernel.
- Orders 5 to 8 (order 0 = full order at n_levels <= 8) and deeper
  truncations (n_levels 16 to 32 at order 1, up to 16 at order 2): fused
  instantiations.  Orders above 8: the plain kernels.

Bars: FP64 inputs 1e-9 relative per entry; FP32 inputs 1e-5 (forward) and
1e-4 per coordinate for gradients, relative to max(|ref|, 1e-2 max |ref|).
"""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle as O
from oracle import ksig_oracle_torch as OT

pytestmark = pytest.mark.gpu


def _walks(rng, n, L, d, scale=0.2):
  return np.cumsum(rng.standard_normal((n, L, d)) * scale, axis=1)


def _rel(a, b):
  a = np.asarray(a, dtype=np.float64)
  b = np.asarray(b, dtype=np.float64)
  return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _grad_err(g, r):
  g = np.asarray(g, dtype=np.float64)
  r = np.asarray(r, dtype=np.float64)
  floor = 1e-2 * np.max(np.abs(r))
  return float(np.max(np.abs(g - r) / np.maximum(np.abs(r), floor)))


@pytest.mark.parametrize('dt,tol', [(np.float64, 1e-9), (np.float32, 1e-5)])
@pytest.mark.parametrize('d', [40, 96])
def test_wide_forward_chunked(dt, tol, d, monkeypatch):
  """d > 32 through the Gram-input sweep, several strips per pair and a
  Gram budget small enough to split the call into several chunks."""
  import ksig_b200 as K
  monkeypatch.setenv('KSIG_GRAM_MB', '1')
  rng = np.random.default_rng(d)
  X = _walks(rng, 7, 300, d).astype(dt)
  Y = _walks(rng, 5, 260, d).astype(dt)
  bw = float(np.sqrt(d) * 0.5)
  for order, m in ((1, 5), (2, 4)):
    k = K.SignatureKernel(n_levels=m, order=order, normalize=True,
                          static_kernel=K.RBFKernel(bw))
    X64, Y64 = X.astype(np.float64), Y.astype(np.float64)
    assert _rel(k(X, Y), O.signature_kernel(X64, Y64, n_levels=m, order=order,
                                            param=bw)) < tol
    assert _rel(k(X), O.signature_kernel(X64, None, n_levels=m, order=order,
                                         param=bw)) < tol
  kp = K.SignaturePDEKernel(dyadic_order=1, normalize=True,
                            static_kernel=K.RBFKernel(bw))
  ref = O.signature_pde_kernel(X.astype(np.float64), Y.astype(np.float64),
                               normalize=True, param=bw, dyadic_order=1)
  assert _rel(kp(X, Y), ref) < (1e-9 if dt == np.float64 else 1e-4)


def test_wide_forward_ragged_ordered():
  """A ragged batch of >= 2048 pairs (longest-first task order) at d = 40."""
  import ksig_b200 as K
  rng = np.random.default_rng(7)
  xs = [np.cumsum(rng.standard_normal((int(L), 40)) * 0.2, 0).astype(np.float32)
        for L in rng.integers(2, 60, 64)]
  ys = [np.cumsum(rng.standard_normal((int(L), 40)) * 0.2, 0).astype(np.float32)
        for L in rng.integers(2, 60, 40)]
  k = K.SignatureKernel(n_levels=4, order=1, normalize=True,
                        static_kernel=K.RBFKernel(3.0))
  ref = O.signature_kernel([x.astype(np.float64) for x in xs],
                           [y.astype(np.float64) for y in ys], n_levels=4, param=3.0)
  assert _rel(k(xs, ys), ref) < 1e-5


def _grad_case(kern_fn, oracle_fn, X, Y, dt, tol):
  import ksig_b200 as K
  Xt = torch.tensor(X, dtype=dt, device='cuda', requires_grad=True)
  Yt = torch.tensor(Y, dtype=dt, device='cuda')
  out = kern_fn(K)(Xt, Yt)
  W = torch.tensor(np.random.default_rng(1).standard_normal(tuple(out.shape)),
                   device='cuda', dtype=out.dtype)
  (out * W).sum().backward()
  Xo = [torch.tensor(x, dtype=torch.float64, requires_grad=True)
        for x in Xt.detach().double().cpu().numpy()]
  Yo = [torch.tensor(y, dtype=torch.float64) for y in Yt.detach().double().cpu().numpy()]
  ref = oracle_fn(Xo, Yo)
  assert _rel(out.detach().cpu().numpy(), ref.detach().numpy()) < (
      1e-9 if dt == torch.float64 else 1e-5)
  (ref * W.double().cpu()).sum().backward()
  g = Xt.grad.cpu().numpy()
  r = torch.stack([x.grad for x in Xo]).numpy()
  assert _grad_err(g, r) < tol, _grad_err(g, r)


@pytest.mark.parametrize('dt,tol', [(torch.float64, 1e-8), (torch.float32, 1e-4)])
@pytest.mark.parametrize('n_levels,order,d', [
    (6, 0, 3),     # full order 6: fused order-6 instantiations
    (8, 5, 3),     # order 5
    (16, 1, 3),    # 16 levels, order 1
    (12, 2, 3),    # 12 levels, order 2
    (10, 0, 2),    # full order 10: plain kernels
    (4, 1, 40),    # 40 channels: Gram-input forward, plain adjoint
    (4, 2, 48),
])
def test_coverage_gradients(dt, tol, n_levels, order, d):
  rng = np.random.default_rng(n_levels * 13 + order + d)
  L1, L2 = (9, 7) if n_levels >= 10 else (21, 17)
  X = _walks(rng, 3, L1, d, 0.3)
  Y = _walks(rng, 2, L2, d, 0.3)
  bw = 0.9 if d < 10 else float(np.sqrt(d) * 0.4)
  _grad_case(
      lambda K: K.SignatureKernel(n_levels=n_levels, order=order, normalize=True,
                                  static_kernel=K.RBFKernel(bw)),
      lambda x, y: OT.signature_kernel(x, y, n_levels=n_levels, order=order,
                                       normalize=True, param=bw),
      X, Y, dt, tol)


@pytest.mark.parametrize('tc', ['1', '0'])
@pytest.mark.parametrize('d', [9, 16, 64])
def test_gram_input_forms_match_oracle(tc, d, monkeypatch):
  """The Gram-input sweep with the tensor-core (tcgen05, 3xTF32) or the
  CUDA-core Gram tiles, forced at widths where a register tile exists too
  (KSIG_FORCE_GIN), on random walks of 200 points (FP32, 1e-5)."""
  import ksig_b200 as K
  monkeypatch.setenv('KSIG_FORCE_GIN', '1')
  monkeypatch.setenv('KSIG_GRAM_TC', tc)
  rng = np.random.default_rng(d + 100)
  inc = rng.standard_normal((6, 199, d)) / np.sqrt(200)
  X = np.concatenate([np.zeros((6, 1, d)), np.cumsum(inc, 1)], 1).astype(np.float32)
  inc = rng.standard_normal((5, 179, d)) / np.sqrt(180)
  Y = np.concatenate([np.zeros((5, 1, d)), np.cumsum(inc, 1)], 1).astype(np.float32)
  bw = float(np.sqrt(d))
  k = K.SignatureKernel(n_levels=5, order=1, normalize=True, static_kernel=K.RBFKernel(bw))
  ref = O.signature_kernel(X.astype(np.float64), Y.astype(np.float64), n_levels=5, param=bw)
  assert _rel(k(X, Y), ref) < 1e-5
  refx = O.signature_kernel(X.astype(np.float64), None, n_levels=5, param=bw)
  assert _rel(k(X), refx) < 1e-5


@pytest.mark.parametrize('d', [128, 160])
def test_wide_spread_walks(d):
  """Widely spread walks (steps of 0.2 per channel) at 128 and 160
  coordinates through the default Gram-input path (CUDA-core difference
  tiles), FP32 against the FP64 oracle at 1e-5, normalised and not."""
  import ksig_b200 as K
  rng = np.random.default_rng(d + 7)
  X = _walks(rng, 4, 45, d).astype(np.float32)
  Y = _walks(rng, 3, 38, d).astype(np.float32)
  bw = float(np.sqrt(d) * 0.5)
  X64, Y64 = X.astype(np.float64), Y.astype(np.float64)
  for normalize, order, m in ((True, 1, 5), (False, 2, 4)):
    k = K.SignatureKernel(n_levels=m, order=order, normalize=normalize,
                          static_kernel=K.RBFKernel(bw))
    assert _rel(k(X, Y), O.signature_kernel(X64, Y64, n_levels=m, order=order,
                                            normalize=normalize, param=bw)) < 1e-5
    assert _rel(k(X), O.signature_kernel(X64, None, n_levels=m, order=order,
                                         normalize=normalize, param=bw)) < 1e-5
