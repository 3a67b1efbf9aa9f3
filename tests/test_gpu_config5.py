"""FP32 parity at the scale of the large ragged workload: N(0, 1) increments
cumsummed over up to 1024 points in d = 16 channels, RBF bandwidth 4,
n_levels = 8, order = 2 (Alg. 6, ksig/algorithms.py:88-140), normalised
(ksig/kernels.py:180-214).  Unnormalised walks of this length reach
|x|^2 ~ 1e4, where the static kernel's |x|^2 + |y|^2 - 2<x, y> cancels in
FP32; the sample holds the longest sequences and their diagonal passes.

Bars, per result, against the FP64 oracle on the same FP32-rounded inputs:
  - normalised K(X, Y) and K(X): relative error <= 1e-5 per entry;
  - per-level kernels: |err| <= 1e-5 * max |level| per level;
  - dX through the adjoint against autograd through the FP64 torch oracle:
    |err_i| <= 1e-4 * max(|ref_i|, 1e-2 * max_j |ref_j|) per coordinate
    (entries smaller than 1 % of the largest are held to 1e-6 of it).
The same gradient bar applies at the 512 x 512 bench shape (L = 200,
d = 8 + time, bandwidth sqrt(8), n_levels = 5, order 1).
"""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle as O
from oracle import ksig_oracle_torch as OT

pytestmark = pytest.mark.gpu

D, BW, M, P = 16, 4.0, 8, 2
FWD_TOL = 1e-5
GRAD_TOL = 1e-4
GRAD_FLOOR = 1e-2


def _walk(rng, L, d=D):
  return np.cumsum(rng.standard_normal((L, d)), 0).astype(np.float32)


def _rel(a, b):
  a = np.asarray(a, dtype=np.float64)
  b = np.asarray(b, dtype=np.float64)
  return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _grad_err(g, r):
  """max_i |g_i - r_i| / max(|r_i|, GRAD_FLOOR * max|r|)."""
  g = np.asarray(g, dtype=np.float64)
  r = np.asarray(r, dtype=np.float64)
  floor = GRAD_FLOOR * np.max(np.abs(r))
  return float(np.max(np.abs(g - r) / np.maximum(np.abs(r), floor)))


def _f64(seqs):
  return [s.astype(np.float64) for s in seqs]


@pytest.fixture(scope='module')
def sample():
  rng = np.random.default_rng(5)
  X = [_walk(rng, L) for L in (1024, 1000, 611, 257, 33)]
  Y = [_walk(rng, L) for L in (1021, 702, 129, 40)]
  return X, Y


def test_config5_forward_normalised(sample):
  import ksig_b200 as K
  X, Y = sample
  k = K.SignatureKernel(n_levels=M, order=P, normalize=True,
                        static_kernel=K.RBFKernel(BW))
  got = k(X, Y)
  ref = O.signature_kernel(_f64(X), _f64(Y), n_levels=M, order=P, param=BW)
  assert got.dtype == np.float32
  assert _rel(got, ref) < FWD_TOL, _rel(got, ref)
  gx = k(X)
  refx = O.signature_kernel(_f64(X), None, n_levels=M, order=P, param=BW)
  assert _rel(gx, refx) < FWD_TOL, _rel(gx, refx)
  # The Ragged form (one padded tensor + lengths) gives the same values.
  Lm = max(s.shape[0] for s in X)
  data = np.zeros((len(X), Lm, D), np.float32)
  for i, s in enumerate(X):
    data[i, :s.shape[0]] = s
  lens = np.array([s.shape[0] for s in X], np.int32)
  gr = k(K.Ragged(torch.as_tensor(data, device='cuda'),
                  torch.as_tensor(lens, device='cuda')), Y)
  assert _rel(gr, ref) < FWD_TOL


def test_config5_levels(sample):
  """Per-level kernels of the longest pairs, including the self pairs that
  feed the normalisation."""
  from ksig_b200 import _engine as E, _lib as Lb
  X, Y = sample
  xs = X[:2] + Y[:1]
  Lm = max(s.shape[0] for s in xs)
  data = np.zeros((len(xs), Lm, D), np.float32)
  for i, s in enumerate(xs):
    data[i, :s.shape[0]] = s
  lens = torch.tensor([s.shape[0] for s in xs], dtype=torch.int32, device='cuda')
  S = E.Seqs(torch.as_tensor(data, device='cuda'), lens)
  got = E.sig_levels(S, S, Lb.PAIRS_FULL, M, P, True, Lb.STATIC_RBF, BW)
  got = got.cpu().numpy().reshape(M + 1, len(xs), len(xs))
  Z = [[O.second_difference(O.static_gram(a, b, 'rbf', BW)) for b in _f64(xs)]
       for a in _f64(xs)]
  ref = np.stack([np.stack([O.sig_levels(z, M, P) for z in row], -1) for row in Z], -2)
  for lev in range(1, M + 1):
    err = np.max(np.abs(got[lev] - ref[lev])) / np.max(np.abs(ref[lev]))
    assert err < FWD_TOL, (lev, err)


def test_config5_input_gradient(sample):
  import ksig_b200 as K
  X, Y = sample
  Xs, Ys = X[:2] + X[3:4], Y[:2]
  Xt = [torch.tensor(s, device='cuda', requires_grad=True) for s in Xs]
  Yt = [torch.tensor(s, device='cuda') for s in Ys]
  k = K.SignatureKernel(n_levels=M, order=P, normalize=True,
                        static_kernel=K.RBFKernel(BW))
  out = k(Xt, Yt, return_on_gpu=True)
  W = torch.tensor(np.random.default_rng(9).standard_normal(tuple(out.shape)),
                   device='cuda', dtype=out.dtype)
  (out * W).sum().backward()
  Xo = [torch.tensor(s, dtype=torch.float64, requires_grad=True) for s in _f64(Xs)]
  Yo = [torch.tensor(s, dtype=torch.float64) for s in _f64(Ys)]
  ref = OT.signature_kernel(Xo, Yo, n_levels=M, order=P, normalize=True, param=BW)
  assert _rel(out.detach().cpu().numpy(), ref.detach().numpy()) < FWD_TOL
  (ref * W.double().cpu()).sum().backward()
  for a, b in zip(Xt, Xo):
    err = _grad_err(a.grad.cpu().numpy(), b.grad.numpy())
    assert err < GRAD_TOL, err


def _bench_walks(rng, n, L, d):
  inc = rng.standard_normal((n, L - 1, d)) / np.sqrt(L)
  X = np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1)
  t = np.broadcast_to(np.linspace(0, 1, L)[None, :, None], (n, L, 1))
  return np.concatenate([X, t], -1).astype(np.float32)


@pytest.mark.parametrize('sym', [False, True])
def test_bench_shape_input_gradient(sym):
  """Per-coordinate dX at the 512 x 512 bench shape, on a 3 x 2 sample."""
  import ksig_b200 as K
  rng = np.random.default_rng(2)
  X = _bench_walks(rng, 3, 200, 8)
  Y = _bench_walks(rng, 2, 200, 8)
  bw = float(np.sqrt(8))
  k = K.SignatureKernel(n_levels=5, order=1, normalize=True,
                        static_kernel=K.RBFKernel(bw))
  Xt = torch.tensor(X, device='cuda', requires_grad=True)
  out = k(Xt) if sym else k(Xt, torch.tensor(Y, device='cuda'))
  W = torch.tensor(np.random.default_rng(4).standard_normal(tuple(out.shape)),
                   device='cuda', dtype=out.dtype)
  (out * W).sum().backward()
  Xo = [torch.tensor(s, dtype=torch.float64, requires_grad=True) for s in X.astype(np.float64)]
  Yo = None if sym else [torch.tensor(s, dtype=torch.float64) for s in Y.astype(np.float64)]
  ref = OT.signature_kernel(Xo, Yo, n_levels=5, order=1, normalize=True, param=bw)
  assert _rel(out.detach().cpu().numpy(), ref.detach().numpy()) < FWD_TOL
  (ref * W.double().cpu()).sum().backward()
  g = Xt.grad.cpu().numpy()
  r = torch.stack([x.grad for x in Xo]).numpy()
  err = _grad_err(g, r)
  assert err < GRAD_TOL, err
