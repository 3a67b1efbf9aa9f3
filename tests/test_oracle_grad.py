"""Pins the FP64 torch oracle: values equal the NumPy oracle, and autograd
gradients equal central finite differences (h = 1e-6, 16 coordinates)."""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle as O
from oracle import ksig_oracle_torch as OT


def _data(seed, nx, ny, lx, ly, d):
  rng = np.random.default_rng(seed)
  xs = [np.cumsum(rng.standard_normal((l, d)) * 0.3, 0) for l in lx[:nx]]
  ys = [np.cumsum(rng.standard_normal((l, d)) * 0.3, 0) for l in ly[:ny]]
  return xs, ys


@pytest.mark.parametrize('kind', ['rbf', 'linear'])
def test_torch_oracle_matches_numpy(kind):
  xs, ys = _data(0, 3, 2, [6, 9, 4], [7, 5], 2)
  tx = [torch.tensor(x) for x in xs]
  ty = [torch.tensor(y) for y in ys]
  for order in (1, 2, 3):
    a = OT.signature_kernel(tx, ty, n_levels=4, order=order, kind=kind,
                            param=0.7).numpy()
    b = O.signature_kernel(xs, ys, n_levels=4, order=order, kind=kind,
                           param=0.7)
    np.testing.assert_allclose(a, b, rtol=1e-12)
  for dy in (0, 1):
    a = OT.signature_pde_kernel(tx, ty, kind=kind, param=0.7,
                                dyadic_order=dy).numpy()
    b = O.signature_pde_kernel(xs, ys, kind=kind, param=0.7, dyadic_order=dy)
    np.testing.assert_allclose(a, b, rtol=1e-12)


def _fd_check(fn, tensors, n_coords=16, h=1e-6, seed=0):
  rng = np.random.default_rng(seed)
  out = fn()
  w = torch.tensor(rng.standard_normal(out.shape))
  loss = (out * w).sum()
  grads = torch.autograd.grad(loss, tensors)
  for _ in range(n_coords):
    ti = rng.integers(len(tensors))
    t = tensors[ti]
    idx = tuple(int(rng.integers(s)) for s in t.shape)
    with torch.no_grad():
      old = t[idx].item()
      t[idx] = old + h
      fp = (fn() * w).sum().item()
      t[idx] = old - h
      fm = (fn() * w).sum().item()
      t[idx] = old
    fd = (fp - fm) / (2 * h)
    an = grads[ti][idx].item()
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (fd, an)


@pytest.mark.parametrize('order', [1, 2])
def test_dp_autograd_vs_finite_differences(order):
  xs, ys = _data(1, 2, 2, [7, 5], [6, 8], 2)
  tx = [torch.tensor(x, requires_grad=True) for x in xs]
  ty = [torch.tensor(y, requires_grad=True) for y in ys]
  bw = torch.tensor(0.8, dtype=torch.float64, requires_grad=True)
  fn = lambda: OT.signature_kernel(tx, ty, n_levels=4, order=order,  # noqa: E731
                                   normalize=True, param=bw)
  _fd_check(fn, tx + ty + [bw])


def test_pde_autograd_vs_finite_differences():
  xs, ys = _data(2, 2, 2, [6, 5], [5, 7], 2)
  tx = [torch.tensor(x, requires_grad=True) for x in xs]
  ty = [torch.tensor(y, requires_grad=True) for y in ys]
  bw = torch.tensor(0.9, dtype=torch.float64, requires_grad=True)
  fn = lambda: OT.signature_pde_kernel(tx, ty, normalize=True, param=bw,  # noqa: E731
                                       dyadic_order=1)
  _fd_check(fn, tx + ty + [bw])
