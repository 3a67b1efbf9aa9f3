"""FP32 parity at wide inputs (d = 20 and 32, padded to 24 and 32
coordinates) with sequences long enough for the planners to reach for wide
tiles.  Above 16 coordinates the library builds no 7/8-column forward tiles
and no 7/8-column (4-column above 16) adjoint tiles, so these shapes run on
the narrower widths, several strips per pair; the results must not change.
Forward against the FP64 oracle, gradients against autograd through the
FP64 torch oracle, on the same rounded inputs.

Bars: forward 1e-5 (DP) / 1e-4 (PDE) relative to the largest entry of the
result; gradients 1e-4 normwise (max |err| / max |ref| per tensor)."""
import numpy as np
import pytest
import torch

from oracle import ksig_oracle as O
from oracle import ksig_oracle_torch as OT

pytestmark = pytest.mark.gpu

DP_TOL = 1e-5
PDE_TOL = 1e-4
GRAD_TOL = 1e-4


def _walks(rng, n, L, d):
  inc = rng.standard_normal((n, L - 1, d)) / np.sqrt(L)
  return np.concatenate([np.zeros((n, 1, d)), np.cumsum(inc, 1)], 1).astype(np.float32)


def _relerr(a, b):
  a = np.asarray(a.detach().cpu() if torch.is_tensor(a) else a, dtype=np.float64)
  b = np.asarray(b.detach().cpu() if torch.is_tensor(b) else b, dtype=np.float64)
  return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize('d', [20, 32])
@pytest.mark.parametrize('order,n_levels', [(1, 5), (2, 4)])
def test_dp_forward_wide(d, order, n_levels):
  import ksig_b200 as K
  rng = np.random.default_rng(300 + d + order)
  X = _walks(rng, 3, 150, d)
  Y = _walks(rng, 2, 230, d)
  bw = float(np.sqrt(d))
  k = K.SignatureKernel(n_levels=n_levels, order=order, normalize=True,
                        static_kernel=K.RBFKernel(bw))
  ref = O.signature_kernel(X.astype(np.float64), Y.astype(np.float64), n_levels=n_levels,
                           order=order, param=bw)
  assert _relerr(k(X, Y), ref) < DP_TOL
  refx = O.signature_kernel(X.astype(np.float64), None, n_levels=n_levels, order=order,
                            param=bw)
  assert _relerr(k(X), refx) < DP_TOL


@pytest.mark.parametrize('d', [20, 32])
@pytest.mark.parametrize('dyadic', [0, 1])
def test_pde_forward_wide(d, dyadic):
  import ksig_b200 as K
  rng = np.random.default_rng(400 + d + dyadic)
  X = _walks(rng, 2, 150, d)
  Y = _walks(rng, 2, 270, d)
  bw = float(np.sqrt(d))
  k = K.SignaturePDEKernel(dyadic_order=dyadic, normalize=True, static_kernel=K.RBFKernel(bw))
  ref = O.signature_pde_kernel(X.astype(np.float64), Y.astype(np.float64), normalize=True,
                               param=bw, dyadic_order=dyadic)
  assert _relerr(k(X, Y), ref) < PDE_TOL


@pytest.mark.parametrize('d', [20, 32])
def test_global_alignment_wide(d):
  import ksig_b200 as K
  rng = np.random.default_rng(500 + d)
  X = _walks(rng, 2, 140, d)
  Y = _walks(rng, 2, 300, d)
  # Global alignment values shrink geometrically with the lengths; a wide
  # bandwidth keeps them inside the FP32 range (about 1e-20 here).
  bw = float(8.0 * np.sqrt(d))
  k = K.GlobalAlignmentKernel(static_kernel=K.RBFKernel(bw))
  ref = O.global_align_kernel(X.astype(np.float64), Y.astype(np.float64), kind='rbf',
                              param=bw)
  assert _relerr(k(X, Y), ref) < PDE_TOL


@pytest.mark.parametrize('d', [20, 32])
@pytest.mark.parametrize('pde', [False, True])
def test_gradients_wide(d, pde):
  import ksig_b200 as K
  rng = np.random.default_rng(600 + d + int(pde))
  # (the FP64 torch oracle of the PDE runs cell by cell: shorter there)
  X = _walks(rng, 2, 60 if pde else 140, d)
  Y = _walks(rng, 2, 90 if pde else 150, d)
  bw = float(np.sqrt(d))
  Xt = torch.tensor(X, device='cuda', requires_grad=True)
  Yt = torch.tensor(Y, device='cuda', requires_grad=True)
  static = K.RBFKernel(bw)
  kern = (K.SignaturePDEKernel(dyadic_order=0, static_kernel=static) if pde else
          K.SignatureKernel(n_levels=4, order=1, static_kernel=static))
  out = kern(Xt, Yt)
  W = torch.tensor(np.random.default_rng(7).standard_normal(tuple(out.shape)),
                   device='cuda', dtype=out.dtype)
  (out * W).sum().backward()
  Xo = [torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in X]
  Yo = [torch.tensor(y, dtype=torch.float64, requires_grad=True) for y in Y]
  ref = (OT.signature_pde_kernel(Xo, Yo, param=bw) if pde else
         OT.signature_kernel(Xo, Yo, n_levels=4, order=1, param=bw))
  assert _relerr(out, ref) < (PDE_TOL if pde else DP_TOL)
  (ref * W.double().cpu()).sum().backward()
  assert _relerr(Xt.grad, torch.stack([x.grad for x in Xo])) < GRAD_TOL
  assert _relerr(Yt.grad, torch.stack([y.grad for y in Yo])) < GRAD_TOL
