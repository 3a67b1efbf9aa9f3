"""Visiting orders of the forward sweep on full pair grids.

Equal-length full grids and K(X) upper triangles run in column-major blocks
per warp, and on full grids the DP levels of one column's pairs in a block
run stacked as one item (separator rows between the row sequences fold each
pair).  Each pair is computed by
one warp with the same arithmetic whatever the order, so the per-level
results must be bit-identical to the round-robin order without stacking.
The grids are large enough that every warp gets pairs from more than one
column, and short enough (17 points) to reach the smallest stacked length.
"""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle as O

pytestmark = pytest.mark.gpu


def _walks(rng, n, L, d):
  inc = rng.standard_normal((n, L - 1, d)) / np.sqrt(L)
  return np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1)


def _levels(X, Y, n_levels, order, monkeypatch, stack, visit):
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as L
  monkeypatch.setenv('KSIG_STACK', stack)
  monkeypatch.setenv('KSIG_VISIT', visit)
  return E.sig_levels(E.Seqs(X), E.Seqs(Y), L.PAIRS_FULL, n_levels, order, True,
                      L.STATIC_RBF, 0.9)


@pytest.mark.parametrize('dt', [torch.float32, torch.float64])
@pytest.mark.parametrize('order,n_levels,nx,lx,ny,ly', [
    (1, 5, 300, 17, 77, 50),
    (1, 3, 131, 33, 97, 120),
    (2, 4, 260, 24, 45, 70),
    (1, 4, 1000, 40, 3, 60),
])
def test_stacked_pairs_bit_identical(dt, order, n_levels, nx, lx, ny, ly, monkeypatch):
  rng = np.random.default_rng(nx + lx + order)
  X = torch.tensor(_walks(rng, nx, lx, 3), dtype=dt, device='cuda')
  Y = torch.tensor(_walks(rng, ny, ly, 3), dtype=dt, device='cuda')
  ref = _levels(X, Y, n_levels, order, monkeypatch, '0', '0')
  blocks = _levels(X, Y, n_levels, order, monkeypatch, '0', '1')
  stacked = _levels(X, Y, n_levels, order, monkeypatch, '1', '1')
  assert torch.equal(blocks, ref)
  assert torch.equal(stacked, ref)
  # A few pairs against the oracle (the stacked rows of neighbouring pairs
  # must not leak into each other).
  Xn, Yn = X.double().cpu().numpy(), Y.double().cpu().numpy()
  for a, b in ((0, 0), (nx - 1, ny - 1), (nx // 2, ny // 3)):
    want = O.signature_kernel(Xn[a:a + 1], Yn[b:b + 1], n_levels=n_levels, order=order,
                              normalize=False, param=0.9)[0, 0]
    got = float(stacked[:, a * ny + b].sum())
    tol = 1e-5 if dt == torch.float32 else 1e-11
    assert abs(got - want) <= tol * abs(want)


@pytest.mark.parametrize('dt', [torch.float32, torch.float64])
@pytest.mark.parametrize('n,lx,n_levels', [(300, 33, 5), (1000, 17, 4), (77, 50, 3), (5, 20, 5)])
def test_stacked_upper_triangle_bit_identical(dt, n, lx, n_levels, monkeypatch):
  """K(X): column-major blocks over the upper triangle (column b holds rows
  0 .. b) against the round-robin order (KSIG_STACK=1 must leave the
  triangle unstacked and unchanged); the output slots keep the row-major
  upper-triangle order."""
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as L
  rng = np.random.default_rng(n + lx)
  X = torch.tensor(_walks(rng, n, lx, 3), dtype=dt, device='cuda')

  def levels(stack, visit):
    monkeypatch.setenv('KSIG_STACK', stack)
    monkeypatch.setenv('KSIG_VISIT', visit)
    return E.sig_levels(E.Seqs(X), None, L.PAIRS_UPPER, n_levels, 1, True, L.STATIC_RBF, 0.9)

  ref = levels('0', '0')
  assert torch.equal(levels('0', '1'), ref)
  stacked = levels('1', '1')
  assert torch.equal(stacked, ref)
  Xn = X.double().cpu().numpy()
  tot = stacked.sum(0).cpu().numpy()
  for a, b in ((0, n - 1), (n // 2, n // 2), (n - 2, n - 1)):
    want = O.signature_kernel(Xn[a:a + 1], Xn[b:b + 1], n_levels=n_levels, normalize=False,
                              param=0.9)[0, 0]
    got = tot[a * n - a * (a - 1) // 2 + (b - a)]
    tol = 1e-5 if dt == torch.float32 else 1e-11
    assert abs(got - want) <= tol * abs(want)


@pytest.mark.parametrize('static', ['linear', 'poly', 'matern32', 'rq'])
def test_stacked_pairs_other_static_kernels(static, monkeypatch):
  """The other static kernels (their own sweep instantiations, which take the
  general step with the run-time epilogue) through the public API on a full
  grid with several pairs per warp: stacked and round-robin orders agree
  bit for bit."""
  import ksig_b200 as K
  sk = {'linear': lambda: K.LinearKernel(0.7),
        'poly': lambda: K.PolynomialKernel(degree=2, gamma=0.5, scale=1.0),
        'matern32': lambda: K.Matern32Kernel(1.3),
        'rq': lambda: K.RationalQuadraticKernel(1.1, 2.0)}[static]()
  rng = np.random.default_rng(17)
  X = _walks(rng, 300, 24, 3).astype(np.float32)
  Y = _walks(rng, 41, 40, 3).astype(np.float32)
  kern = K.SignatureKernel(n_levels=4, order=1, normalize=False, static_kernel=sk)
  monkeypatch.setenv('KSIG_STACK', '0')
  monkeypatch.setenv('KSIG_VISIT', '0')
  ref = kern(X, Y)
  monkeypatch.setenv('KSIG_STACK', '1')
  monkeypatch.setenv('KSIG_VISIT', '1')
  assert np.array_equal(kern(X, Y), ref)


def test_stacked_pairs_bench_size(monkeypatch):
  """The bench workload at full size (512 x 512 pairs, L = 200, d = 8 + time,
  m = 5, RBF): stacked, blocked and round-robin orders give the same levels
  bit for bit, and sampled pairs match the FP64 oracle."""
  import bench
  X = torch.as_tensor(bench.make_walks(512, 200, 8, 2), device='cuda')
  Y = torch.as_tensor(bench.make_walks(512, 200, 8, 3), device='cuda')
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as L

  def levels(stack, visit):
    monkeypatch.setenv('KSIG_STACK', stack)
    monkeypatch.setenv('KSIG_VISIT', visit)
    return E.sig_levels(E.Seqs(X), E.Seqs(Y), L.PAIRS_FULL, 5, 1, True, L.STATIC_RBF,
                        float(np.sqrt(8)))

  ref = levels('0', '0')
  assert torch.equal(levels('0', '1'), ref)
  stacked = levels('1', '1')
  assert torch.equal(stacked, ref)
  Xn, Yn = X.double().cpu().numpy(), Y.double().cpu().numpy()
  for a, b in ((0, 0), (511, 511), (300, 17), (17, 300)):
    want = O.signature_kernel(Xn[a:a + 1], Yn[b:b + 1], n_levels=5, normalize=False,
                              param=float(np.sqrt(8)))[0, 0]
    got = float(stacked[:, a * 512 + b].sum())
    assert abs(got - want) <= 1e-5 * abs(want)


@pytest.mark.parametrize('dt', [torch.float32, torch.float64])
@pytest.mark.parametrize('nx,lx,ny,ly,dyadic', [
    (300, 17, 77, 50, 0),
    (131, 33, 97, 120, 1),
    (1000, 40, 3, 60, 0),
    (200, 20, 60, 45, 2),
])
def test_stacked_pde_bit_identical(dt, nx, lx, ny, ly, dyadic, monkeypatch):
  """Goursat PDE on full grids: stacked columns (the separator row resets
  the lane's K values to the boundary value) against round-robin pairs, bit
  for bit, and sampled pairs against the FP64 oracle."""
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as L
  rng = np.random.default_rng(nx + ly + dyadic)
  X = torch.tensor(_walks(rng, nx, lx, 3), dtype=dt, device='cuda')
  Y = torch.tensor(_walks(rng, ny, ly, 3), dtype=dt, device='cuda')

  def values(stack):
    monkeypatch.setenv('KSIG_STACK', stack)
    return E.pde_values(E.Seqs(X), E.Seqs(Y), L.PAIRS_FULL, dyadic, True, L.STATIC_RBF, 0.9)

  ref = values('0')
  stacked = values('1')
  assert torch.equal(stacked, ref)
  Xn, Yn = X.double().cpu().numpy(), Y.double().cpu().numpy()
  for a, b in ((0, 0), (nx - 1, ny - 1), (nx // 2, ny // 3)):
    want = O.signature_pde_kernel(Xn[a:a + 1], Yn[b:b + 1], normalize=False,
                                  dyadic_order=dyadic, param=0.9)[0, 0]
    got = float(stacked[a * ny + b])
    tol = 1e-4 if dt == torch.float32 else 1e-10
    assert abs(got - want) <= tol * abs(want)


@pytest.mark.parametrize('static', ['matern32', 'poly'])
def test_pde_other_static_kernels_full_grid(static, monkeypatch):
  """PDE K(X, Y) on a full grid of equal-length sequences with the other
  static kernels (their own sweep instantiations, which have no stacked
  form): the same values with and without stacking enabled, and the FP64
  oracle on sampled pairs."""
  import ksig_b200 as K
  sk = {'matern32': lambda: K.Matern32Kernel(1.3),
        'poly': lambda: K.PolynomialKernel(degree=2, gamma=0.5, scale=1.0)}[static]()
  rng = np.random.default_rng(29)
  X = _walks(rng, 200, 24, 3)
  Y = _walks(rng, 41, 30, 3)
  kern = K.SignaturePDEKernel(normalize=False, static_kernel=sk, dyadic_order=0)
  monkeypatch.setenv('KSIG_STACK', '0')
  ref = kern(X, Y)
  monkeypatch.setenv('KSIG_STACK', '1')
  got = kern(X, Y)
  assert np.array_equal(got, ref)
  param = {'matern32': 1.3, 'poly': (2, 0.5, 1.0)}[static]
  for a, b in ((0, 0), (199, 40), (77, 13)):
    want = O.signature_pde_kernel(X[a:a + 1], Y[b:b + 1], normalize=False, kind=static,
                                  param=param, dyadic_order=0)[0, 0]
    assert abs(got[a, b] - want) <= 1e-9 * abs(want)
