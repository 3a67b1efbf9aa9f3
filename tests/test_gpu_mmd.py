"""Signature-kernel MMD^2 gradients (PDE kernel, dyadic order 2) against
central finite differences in FP64 (h = 1e-6) on 16 random coordinates and
on the RBF bandwidth, the check the gradient workload asks for.  The
finite differences evaluate this library's own FP64 forward, which the
oracle tests pin to the reference."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _paths(rng, n, L, d, drift_sd):
  drift = rng.standard_normal((n, 1, d)) * drift_sd
  inc = rng.standard_normal((n, L - 1, d)) / np.sqrt(L) + drift / L
  return np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1)


def _mmd2(kern, X, Y):
  kxx = kern(X, return_on_gpu=True)
  kyy = kern(Y, return_on_gpu=True)
  kxy = kern(X, Y, return_on_gpu=True)
  return kxx.mean() + kyy.mean() - 2.0 * kxy.mean()


@pytest.mark.parametrize('normalize', [False, True])
def test_mmd2_pde_dyadic2_grad_vs_central_fd(normalize):
  import ksig_b200 as K
  rng = np.random.default_rng(44)
  Xn = _paths(rng, 12, 24, 4, np.sqrt(0.5))
  Yn = _paths(rng, 10, 24, 4, np.sqrt(0.5))
  bw0 = 1.3
  X = torch.tensor(Xn, device='cuda', requires_grad=True)
  Y = torch.tensor(Yn, device='cuda')
  bw = torch.tensor(bw0, dtype=torch.float64, requires_grad=True)
  kern = K.SignaturePDEKernel(dyadic_order=2, normalize=normalize,
                              static_kernel=K.RBFKernel(bw))
  _mmd2(kern, X, Y).backward()
  gX = X.grad.detach().cpu().numpy()
  gb = float(bw.grad)

  def f(Xv, b):
    k = K.SignaturePDEKernel(dyadic_order=2, normalize=normalize,
                             static_kernel=K.RBFKernel(b))
    with torch.no_grad():
      return float(_mmd2(k, torch.tensor(Xv, device='cuda'), Y))

  h = 1e-6
  idx = [tuple(rng.integers(0, s) for s in Xn.shape) for _ in range(16)]
  scale = np.abs(gX).max()
  for i in idx:
    Xp, Xm = Xn.copy(), Xn.copy()
    Xp[i] += h
    Xm[i] -= h
    fd = (f(Xp, bw0) - f(Xm, bw0)) / (2 * h)
    assert abs(fd - gX[i]) <= 1e-4 * scale + 1e-7, (i, fd, gX[i])
  fdb = (f(Xn, bw0 + h) - f(Xn, bw0 - h)) / (2 * h)
  assert abs(fdb - gb) <= 1e-4 * max(1.0, abs(fdb)), (fdb, gb)
