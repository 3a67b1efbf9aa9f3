"""Forward parity of the CUDA kernels against the reference and the oracle.

Tolerances (relative, per result): FP64 inputs run FP64 kernels and must
match the reference goldens to 1e-9; FP32 inputs must match the FP64 oracle
on the same (FP32-rounded) inputs to 1e-5 for the DP kernel and 1e-4 for the
PDE kernel, the bars set for the mixed-precision path.
"""
import numpy as np
import pytest
import torch

from golden_io import load_cases
from oracle import ksig_oracle as O

pytestmark = pytest.mark.gpu

CASES = load_cases()
DP_TOL = 1e-5
PDE_TOL = 1e-4


def _static(K, name, v):
  if name == 'rbf':
    return K.RBFKernel(v)
  if name == 'linear':
    return K.LinearKernel(v)
  if name == 'poly':
    return K.PolynomialKernel(degree=v[0], gamma=v[1], scale=v[2])
  if name == 'matern12':
    return K.Matern12Kernel(v)
  if name == 'matern32':
    return K.Matern32Kernel(v)
  if name == 'matern52':
    return K.Matern52Kernel(v)
  if name == 'rq':
    return K.RationalQuadraticKernel(bandwidth=v[0], alpha=v[1])
  raise ValueError(name)


def _kern(c, **over):
  import ksig_b200 as K
  p = dict(c['params'], **over)
  static = _static(K, p['static'], p['param'])
  if c['kernel'] == 'sig':
    return K.SignatureKernel(
        n_levels=p['n_levels'], order=p['order'],
        difference=p.get('difference', True), normalize=p['normalize'],
        static_kernel=static)
  if c['kernel'] == 'ga':
    return K.GlobalAlignmentKernel(static_kernel=static)
  return K.SignaturePDEKernel(difference=p.get('difference', True),
                              normalize=p['normalize'], static_kernel=static,
                              dyadic_order=p.get('dyadic_order', 0))


def _oracle(c, X, Y=None, diag=False, **over):
  p = dict(c['params'], **over)
  if c['kernel'] == 'sig':
    return O.signature_kernel(
        X, Y, diag=diag, n_levels=p['n_levels'], order=p['order'],
        difference=p.get('difference', True), normalize=p['normalize'],
        kind=p['static'], param=p['param'])
  if c['kernel'] == 'ga':
    return O.global_align_kernel(X, Y, diag=diag, kind=p['static'], param=p['param'])
  return O.signature_pde_kernel(
      X, Y, diag=diag, difference=p.get('difference', True),
      normalize=p['normalize'], kind=p['static'], param=p['param'],
      dyadic_order=p.get('dyadic_order', 0))


def _relerr(a, b):
  a = np.asarray(a, dtype=np.float64)
  b = np.asarray(b, dtype=np.float64)
  return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _cast(X, dt):
  if isinstance(X, list):
    return [np.asarray(x, dtype=dt) for x in X]
  return np.asarray(X, dtype=dt)


@pytest.mark.parametrize('c', CASES, ids=[c['name'] for c in CASES])
def test_golden_fp64(c):
  """FP64 inputs reproduce the reference's own outputs."""
  k = _kern(c)
  X, Y = c['X'], c['Y']
  assert _relerr(k(X), c['KXX']) < 1e-9
  assert _relerr(k(X, Y), c['KXY']) < 1e-9
  assert _relerr(k(X, diag=True), c['Kdiag']) < 1e-9


@pytest.mark.parametrize('c', CASES, ids=[c['name'] for c in CASES])
def test_golden_fp32(c):
  """FP32 inputs against the FP64 oracle on the same rounded inputs."""
  k = _kern(c)
  X32, Y32 = _cast(c['X'], np.float32), _cast(c['Y'], np.float32)
  X64, Y64 = _cast(X32, np.float64), _cast(Y32, np.float64)
  tol = DP_TOL if c['kernel'] == 'sig' else PDE_TOL
  out = k(X32, Y32)
  assert out.dtype == np.float32
  if c['kernel'] == 'ga':
    # Alignment values span hundreds of decades; compare the entries an
    # FP32 output can represent (the rest underflow to 0 as they would in
    # the reference run in FP32).
    def check(a, b):
      m = b > 1e-30
      assert np.all(a[~m] < 1e-28)
      assert _relerr(a[m], b[m]) < tol
    check(out, _oracle(c, X64, Y64))
    check(k(X32), _oracle(c, X64))
    assert _relerr(k(X32, diag=True), _oracle(c, X64, diag=True)) < tol
    return
  assert _relerr(out, _oracle(c, X64, Y64)) < tol
  assert _relerr(k(X32), _oracle(c, X64)) < tol
  assert _relerr(k(X32, diag=True), _oracle(c, X64, diag=True)) < tol


def _walks(rng, n, L, d, time=True, scale=None):
  scale = 1.0 / np.sqrt(L) if scale is None else scale
  inc = rng.standard_normal((n, L - 1, d)) * scale
  X = np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1)
  if time:
    t = np.broadcast_to(np.linspace(0, 1, L)[None, :, None], (n, L, 1))
    X = np.concatenate([X, t], -1)
  return X


def test_config2_shapes_fp32():
  """Random walks + time, L=200, d=8+1, sigma=sqrt(8), m=5, normalize."""
  import ksig_b200 as K
  rng = np.random.default_rng(2)
  X = _walks(rng, 12, 200, 8)
  Y = _walks(rng, 10, 200, 8)
  k = K.SignatureKernel(n_levels=5, order=1, normalize=True,
                        static_kernel=K.RBFKernel(np.sqrt(8)))
  X32, Y32 = X.astype(np.float32), Y.astype(np.float32)
  ref = O.signature_kernel(X32.astype(np.float64), Y32.astype(np.float64),
                           n_levels=5, param=np.sqrt(8))
  assert _relerr(k(X32, Y32), ref) < DP_TOL
  lev = O.signature_kernel(X32.astype(np.float64), Y32.astype(np.float64),
                           n_levels=5, param=np.sqrt(8), return_levels=True)
  from ksig_b200 import _engine as E, _lib as Lb
  Xs = E.Seqs(torch.as_tensor(X32, device='cuda'))
  Ys = E.Seqs(torch.as_tensor(Y32, device='cuda'))
  got = E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, 5, 1, True, Lb.STATIC_RBF,
                     np.sqrt(8)).cpu().numpy().reshape(lev.shape)
  scale = np.abs(lev).max(axis=(1, 2), keepdims=True)
  assert np.max(np.abs(got - lev) / scale) < 1e-5


@pytest.mark.parametrize('dt', [np.float32, np.float64])
@pytest.mark.parametrize('L', [40, 300, 700])
def test_dp_multi_strip_and_lengths(dt, L):
  """Column sequences longer than one strip (boundary hand-over)."""
  import ksig_b200 as K
  rng = np.random.default_rng(L)
  X = _walks(rng, 3, L, 3)
  Y = _walks(rng, 2, L + 37, 3)
  k = K.SignatureKernel(n_levels=4, order=1, normalize=True,
                        static_kernel=K.RBFKernel(0.8))
  ref = O.signature_kernel(X.astype(dt).astype(np.float64),
                           Y.astype(dt).astype(np.float64), n_levels=4,
                           param=0.8)
  tol = DP_TOL if dt == np.float32 else 1e-10
  assert _relerr(k(X.astype(dt), Y.astype(dt)), ref) < tol


@pytest.mark.parametrize('order,n_levels', [(2, 3), (2, 8), (3, 5), (4, 4)])
def test_dp_higher_order_fp32(order, n_levels):
  import ksig_b200 as K
  rng = np.random.default_rng(order * 10 + n_levels)
  X = _walks(rng, 4, 90, 5)
  Y = _walks(rng, 3, 61, 5)
  k = K.SignatureKernel(n_levels=n_levels, order=order, normalize=True,
                        static_kernel=K.RBFKernel(1.1))
  X32, Y32 = X.astype(np.float32), Y.astype(np.float32)
  ref = O.signature_kernel(X32.astype(np.float64), Y32.astype(np.float64),
                           n_levels=n_levels, order=order, param=1.1)
  assert _relerr(k(X32, Y32), ref) < DP_TOL


def test_ragged_dp_and_pde_fp32():
  """Ragged batches equal the per-pair oracle (edge-padding invariance)."""
  import ksig_b200 as K
  rng = np.random.default_rng(7)
  xs = [np.cumsum(rng.standard_normal((n, 4)) * 0.2, 0).astype(np.float32)
        for n in (5, 33, 64, 129, 300, 2)]
  ys = [np.cumsum(rng.standard_normal((n, 4)) * 0.2, 0).astype(np.float32)
        for n in (17, 250, 64, 1)]
  x64 = [x.astype(np.float64) for x in xs]
  y64 = [y.astype(np.float64) for y in ys]
  k = K.SignatureKernel(n_levels=5, order=2, normalize=False,
                        static_kernel=K.RBFKernel(0.9))
  ref = O.signature_kernel(x64, y64, n_levels=5, order=2, normalize=False,
                           param=0.9)
  assert _relerr(k(xs, ys), ref) < DP_TOL
  kp = K.SignaturePDEKernel(normalize=False, static_kernel=K.RBFKernel(0.9),
                            dyadic_order=1)
  refp = O.signature_pde_kernel(x64, y64, normalize=False, param=0.9,
                                dyadic_order=1)
  assert _relerr(kp(xs, ys), refp) < PDE_TOL


@pytest.mark.parametrize('dyadic', [0, 1, 2, 3])
@pytest.mark.parametrize('dt', [np.float32, np.float64])
def test_pde_dyadic(dyadic, dt):
  import ksig_b200 as K
  rng = np.random.default_rng(40 + dyadic)
  X = _walks(rng, 3, 70, 3)
  Y = _walks(rng, 4, 45, 3)
  k = K.SignaturePDEKernel(normalize=True, static_kernel=K.RBFKernel(0.7),
                           dyadic_order=dyadic)
  ref = O.signature_pde_kernel(X.astype(dt).astype(np.float64),
                               Y.astype(dt).astype(np.float64), param=0.7,
                               dyadic_order=dyadic)
  tol = PDE_TOL if dt == np.float32 else 1e-10
  assert _relerr(k(X.astype(dt), Y.astype(dt)), ref) < tol


@pytest.mark.parametrize('L', [260, 600])
def test_pde_multi_strip(L):
  import ksig_b200 as K
  rng = np.random.default_rng(L)
  X = _walks(rng, 2, L, 3)
  Y = _walks(rng, 2, L + 5, 3)
  k = K.SignaturePDEKernel(normalize=False, static_kernel=K.RBFKernel(1.0),
                           dyadic_order=1)
  ref = O.signature_pde_kernel(X.astype(np.float32).astype(np.float64),
                               Y.astype(np.float32).astype(np.float64),
                               normalize=False, dyadic_order=1)
  assert _relerr(k(X.astype(np.float32), Y.astype(np.float32)), ref) < PDE_TOL


def test_symmetry_and_diag_consistency():
  """K(X,Y) = K(Y,X)^T and diag(K(X)) = K(X, diag=True) (normalize=False)."""
  import ksig_b200 as K
  rng = np.random.default_rng(9)
  X = _walks(rng, 7, 120, 4).astype(np.float32)
  Y = _walks(rng, 5, 80, 4).astype(np.float32)
  for k in (K.SignatureKernel(n_levels=6, normalize=False),
            K.SignaturePDEKernel(normalize=False, dyadic_order=1)):
    a = k(X, Y)
    b = k(Y, X)
    assert _relerr(a, b.T) < 1e-5
    assert _relerr(np.diag(k(X)), k(X, diag=True)) < 1e-5


def test_return_on_gpu_and_torch_inputs():
  import ksig_b200 as K
  rng = np.random.default_rng(3)
  X = torch.as_tensor(_walks(rng, 4, 30, 2), dtype=torch.float32)
  k = K.SignatureKernel(n_levels=3)
  out = k(X, return_on_gpu=True)
  assert isinstance(out, torch.Tensor) and out.is_cuda
  assert out.dtype == torch.float32
  np.testing.assert_allclose(out.cpu().numpy(), k(X.numpy()), rtol=0, atol=0)


def test_api_errors():
  import ksig_b200 as K
  with pytest.raises(ValueError):
    K.SignatureKernel(n_levels=0)
  with pytest.raises(ValueError):
    K.RBFKernel(bandwidth=-1.0)
  k = K.SignatureKernel(n_levels=2, n_features=3)
  with pytest.raises(ValueError):
    k(np.zeros((2, 4, 2)))
  with pytest.raises(ValueError):
    k(np.zeros((2, 4, 3, 1)))


@pytest.mark.parametrize('order,n_levels', [(1, 5), (2, 4)])
def test_plain_baseline_kernel_matches_oracle(order, n_levels):
  """The plain one-pair-per-block baseline computes the same levels."""
  from ksig_b200 import _engine as E, _lib as Lb
  rng = np.random.default_rng(70 + order)
  X = _walks(rng, 3, 50, 3).astype(np.float32)
  Y = _walks(rng, 4, 37, 3).astype(np.float32)
  ref = O.signature_kernel(X.astype(np.float64), Y.astype(np.float64),
                           n_levels=n_levels, order=order, param=0.8,
                           return_levels=True)
  got = E.sig_levels_plain(E.Seqs(torch.as_tensor(X, device='cuda')),
                           E.Seqs(torch.as_tensor(Y, device='cuda')),
                           Lb.PAIRS_FULL, n_levels, order, Lb.STATIC_RBF, 0.8)
  got = got.cpu().numpy().reshape(ref.shape)
  scale = np.abs(ref).max(axis=(1, 2), keepdims=True)
  assert np.max(np.abs(got - ref) / scale) < 1e-5


@pytest.mark.parametrize('name,param', [('matern12', 0.8), ('matern32', 1.2),
                                        ('matern52', 0.7), ('poly', (2.0, 0.1, 0.2)),
                                        ('rq', (0.9, 0.7))])
@pytest.mark.parametrize('dt,tol', [(np.float64, 1e-9), (np.float32, 1e-5)])
def test_other_static_kernels_vs_oracle(name, param, dt, tol):
  """Every static kernel of ksig.static.kernels, fused into the Gram
  epilogue of the DP and PDE sweeps, against the FP64 oracle (Matern12 / 32
  with the distance between x and y; their reference outputs are not
  usable, see oracle.ksig_oracle.static_gram)."""
  import ksig_b200 as K
  rng = np.random.default_rng(90)
  X = np.cumsum(rng.standard_normal((4, 19, 3)) * 0.3, axis=1).astype(dt)
  Y = np.cumsum(rng.standard_normal((3, 23, 3)) * 0.3, axis=1).astype(dt)
  Xo, Yo = X.astype(np.float64), Y.astype(np.float64)
  for normalize in (False, True):
    sk = _static(K, name, param)
    got = K.SignatureKernel(n_levels=4, order=2, normalize=normalize, static_kernel=sk)(X, Y)
    ref = O.signature_kernel(Xo, Yo, n_levels=4, order=2, normalize=normalize,
                             kind=name, param=param)
    assert _relerr(got, ref) < tol, (name, normalize)
    got = K.SignaturePDEKernel(normalize=normalize, static_kernel=sk, dyadic_order=1)(X)
    ref = O.signature_pde_kernel(Xo, None, normalize=normalize, kind=name, param=param,
                                 dyadic_order=1)
    assert _relerr(got, ref) < max(tol, 1e-9 if dt == np.float64 else PDE_TOL), (name, normalize)


def test_other_static_kernels_reject_gradients():
  import ksig_b200 as K
  X = torch.randn((2, 6, 2), dtype=torch.float64, device='cuda', requires_grad=True)
  kern = K.SignatureKernel(n_levels=2, static_kernel=K.Matern52Kernel(1.0))
  with pytest.raises(NotImplementedError):
    kern(X)
  with pytest.raises(ValueError):
    K.RationalQuadraticKernel(bandwidth=1.0, alpha=-1.0)


def test_global_alignment_ragged_multi_strip():
  """Global alignment on ragged batches whose column sequences span several
  strips, FP64 against the oracle and FP32 within the PDE tolerance."""
  import ksig_b200 as K
  rng = np.random.default_rng(95)
  xs = [np.cumsum(rng.standard_normal((n, 2)) * 0.2, 0) for n in (40, 290, 7)]
  ys = [np.cumsum(rng.standard_normal((n, 2)) * 0.2, 0) for n in (300, 12)]
  ref = O.global_align_kernel(xs, ys, kind='rbf', param=0.9)
  refx = O.global_align_kernel(xs, None, kind='rbf', param=0.9)
  kern = K.GlobalAlignmentKernel(static_kernel=K.RBFKernel(0.9))
  assert _relerr(kern(xs, ys), ref) < 1e-9
  assert _relerr(kern(xs), refx) < 1e-9
  got = kern([x.astype(np.float32) for x in xs], [y.astype(np.float32) for y in ys])
  ref32 = O.global_align_kernel([x.astype(np.float32).astype(np.float64) for x in xs],
                                [y.astype(np.float32).astype(np.float64) for y in ys],
                                kind='rbf', param=0.9)
  assert _relerr(got, ref32) < PDE_TOL


@pytest.mark.parametrize('n_levels', [7, 10, 12])
def test_deep_truncation_levels(n_levels):
  """n_levels beyond the common range (the kernels for 10 and 12 levels;
  7 runs the 8-level kernel and drops the top level)."""
  import ksig_b200 as K
  rng = np.random.default_rng(97)
  X = np.cumsum(rng.standard_normal((3, 30, 3)) * 0.3, axis=1)
  Y = np.cumsum(rng.standard_normal((2, 25, 3)) * 0.3, axis=1)
  ref = O.signature_kernel(X, Y, n_levels=n_levels, normalize=True, param=0.7)
  kern = K.SignatureKernel(n_levels=n_levels, static_kernel=K.RBFKernel(0.7))
  assert _relerr(kern(X, Y), ref) < 1e-9
  assert _relerr(kern(X.astype(np.float32), Y.astype(np.float32)),
                 O.signature_kernel(X.astype(np.float32).astype(np.float64),
                                    Y.astype(np.float32).astype(np.float64),
                                    n_levels=n_levels, normalize=True, param=0.7)) < DP_TOL


@pytest.mark.parametrize('d', [5, 7, 10, 11, 15])
@pytest.mark.parametrize('order', [1, 2])
def test_paired_gram_widths_fp32(d, order):
  """FP32 instances whose Gram runs as paired FFMA2 over coordinate pairs
  (7-column order-1 and 4-column order-2 tiles with n_levels >= 5): odd and
  even padded widths (6, 8, 10, 12, 16)."""
  import ksig_b200 as K
  rng = np.random.default_rng(700 + d + 10 * order)
  X = _walks(rng, 3, 200, d, time=False)
  Y = _walks(rng, 2, 190, d, time=False)
  bw = float(np.sqrt(d))
  k = K.SignatureKernel(n_levels=5, order=order, normalize=True,
                        static_kernel=K.RBFKernel(bw))
  X32, Y32 = X.astype(np.float32), Y.astype(np.float32)
  ref = O.signature_kernel(X32.astype(np.float64), Y32.astype(np.float64),
                           n_levels=5, order=order, param=bw)
  assert _relerr(k(X32, Y32), ref) < DP_TOL
