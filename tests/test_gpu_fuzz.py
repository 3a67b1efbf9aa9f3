"""Seeded random sweep over shapes, orders, level counts, refinements,
static kernels, ragged lengths and strip counts: every combination the
dispatch can reach, against the FP64 oracle (forward) and the FP64 torch
oracle under autograd (gradients).  FP64 inputs, so the bar is 1e-9 (1e-8 for
gradients); the cases are small enough for the oracle."""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle as O
from oracle import ksig_oracle_torch as OT

pytestmark = pytest.mark.gpu


def _rel(a, b):
  a = np.asarray(a, dtype=np.float64)
  b = np.asarray(b, dtype=np.float64)
  return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _seqs(rng, n, lmin, lmax, d):
  return [np.cumsum(rng.standard_normal((int(L), d)) * 0.25, 0)
          for L in rng.integers(lmin, lmax + 1, n)]


@pytest.mark.parametrize('seed', range(12))
def test_fuzz_forward(seed):
  import ksig_b200 as K
  rng = np.random.default_rng(1000 + seed)
  d = int(rng.choice([1, 2, 3, 5, 8]))
  lmax = int(rng.choice([6, 40, 140]))          # 140 spans several 2-column strips
  xs = _seqs(rng, int(rng.integers(1, 5)), 1, lmax, d)
  ys = _seqs(rng, int(rng.integers(1, 4)), 1, lmax, d)
  bw = float(rng.uniform(0.4, 2.0))
  if seed % 3 == 2:
    dy = int(rng.integers(0, 3))
    kern = K.SignaturePDEKernel(dyadic_order=dy, normalize=bool(seed % 2),
                                static_kernel=K.RBFKernel(bw))
    ref = O.signature_pde_kernel(xs, ys, normalize=bool(seed % 2), param=bw, dyadic_order=dy)
    refx = O.signature_pde_kernel(xs, None, normalize=bool(seed % 2), param=bw,
                                  dyadic_order=dy)
  else:
    m = int(rng.integers(1, 7))
    p = int(rng.integers(1, min(m, 4) + 1))
    kern = K.SignatureKernel(n_levels=m, order=p, normalize=bool(seed % 2),
                             static_kernel=K.RBFKernel(bw))
    ref = O.signature_kernel(xs, ys, n_levels=m, order=p, normalize=bool(seed % 2), param=bw)
    refx = O.signature_kernel(xs, None, n_levels=m, order=p, normalize=bool(seed % 2),
                              param=bw)
  assert _rel(kern(xs, ys), ref) < 1e-9
  assert _rel(kern(xs), refx) < 1e-9


@pytest.mark.parametrize('seed', range(6))
def test_fuzz_gradients(seed):
  import ksig_b200 as K
  rng = np.random.default_rng(2000 + seed)
  d = int(rng.choice([1, 2, 4]))
  n, L = int(rng.integers(1, 4)), int(rng.choice([5, 20, 40]))
  X = np.cumsum(rng.standard_normal((n, L, d)) * 0.25, 1)
  Y = np.cumsum(rng.standard_normal((2, int(rng.choice([4, 30, 50])), d)) * 0.25, 1)
  bw0 = float(rng.uniform(0.5, 1.5))
  pde = seed % 2 == 1
  m = int(rng.integers(2, 6))
  p = int(rng.integers(1, 3))
  dy = int(rng.integers(0, 2))
  Xt = torch.tensor(X, device='cuda', requires_grad=True)
  Yt = torch.tensor(Y, device='cuda', requires_grad=True)
  bt = torch.tensor(bw0, dtype=torch.float64, requires_grad=True)
  kern = (K.SignaturePDEKernel(dyadic_order=dy, static_kernel=K.RBFKernel(bt)) if pde else
          K.SignatureKernel(n_levels=m, order=p, static_kernel=K.RBFKernel(bt)))
  out = kern(Xt, Yt)
  W = torch.tensor(rng.standard_normal(tuple(out.shape)), device='cuda')
  (out * W).sum().backward()
  Xo = [torch.tensor(x, requires_grad=True) for x in X]
  Yo = [torch.tensor(y, requires_grad=True) for y in Y]
  bo = torch.tensor(bw0, dtype=torch.float64, requires_grad=True)
  ref = (OT.signature_pde_kernel(Xo, Yo, dyadic_order=dy, param=bo) if pde else
         OT.signature_kernel(Xo, Yo, n_levels=m, order=p, param=bo))
  (ref * W.cpu()).sum().backward()
  assert _rel(out.detach().cpu(), ref.detach()) < 1e-9
  assert _rel(Xt.grad.cpu(), torch.stack([x.grad for x in Xo])) < 1e-8
  assert _rel(Yt.grad.cpu(), torch.stack([y.grad for y in Yo])) < 1e-8
  assert abs(bt.grad.item() - bo.grad.item()) <= 1e-8 * max(1.0, abs(bo.grad.item()))
