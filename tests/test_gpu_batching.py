"""Ragged batching machinery on the GPU: the longest-first task order, the
Ragged input form, CUDA-graph capture and the tile-width autotuner.  None of
these may change a result: the order only reschedules independent pairs,
the graph replays the same launches, the tuner only picks among compiled
kernels that are each checked against the oracle elsewhere."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ragged(rng, n, lmin, lmax, d, dt=torch.float32):
  lens = rng.integers(lmin, lmax + 1, n)
  data = np.zeros((n, lmax, d))
  for i, L in enumerate(lens):
    data[i, :L] = np.cumsum(rng.standard_normal((L, d)) * 0.3, 0)
  return (torch.tensor(data, dtype=dt, device='cuda'),
          torch.tensor(lens, dtype=torch.int32, device='cuda'))


def _with_order(flag, fn):
  old = os.environ.get('KSIG_TASK_ORDER')
  os.environ['KSIG_TASK_ORDER'] = flag
  try:
    return fn()
  finally:
    if old is None:
      del os.environ['KSIG_TASK_ORDER']
    else:
      os.environ['KSIG_TASK_ORDER'] = old


def test_task_order_changes_no_result():
  from ksig_b200 import _engine as E, _lib as Lb
  rng = np.random.default_rng(3)
  X, lx = _ragged(rng, 48, 3, 40, 3)
  Y, ly = _ragged(rng, 50, 3, 40, 3)   # 2400 pairs: the order is built
  Xs, Ys = E.Seqs(X, lx), E.Seqs(Y, ly)
  for order in (1, 2):
    a = _with_order('0', lambda: E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, 4, order, True,
                                              Lb.STATIC_RBF, 0.8))
    b = _with_order('1', lambda: E.sig_levels(Xs, Ys, Lb.PAIRS_FULL, 4, order, True,
                                              Lb.STATIC_RBF, 0.8))
    assert torch.equal(a, b)
  a = _with_order('0', lambda: E.pde_values(Xs, Ys, Lb.PAIRS_FULL, 1, True, Lb.STATIC_RBF, 0.8))
  b = _with_order('1', lambda: E.pde_values(Xs, Ys, Lb.PAIRS_FULL, 1, True, Lb.STATIC_RBF, 0.8))
  assert torch.equal(a, b)
  gl = torch.tensor(rng.standard_normal((5, 48 * 50)), device='cuda')
  da, pa = _with_order('0', lambda: E.sig_levels_bwd(Xs, Ys, Lb.PAIRS_FULL, 4, 1,
                                                     Lb.STATIC_RBF, 0.8, gl))
  db, pb = _with_order('1', lambda: E.sig_levels_bwd(Xs, Ys, Lb.PAIRS_FULL, 4, 1,
                                                     Lb.STATIC_RBF, 0.8, gl))
  scale = da.abs().max().item()
  assert (da - db).abs().max().item() <= 1e-5 * scale
  assert abs(pa.item() - pb.item()) <= 1e-9 * max(1.0, abs(pa.item()))
  g = torch.tensor(rng.standard_normal(48 * 50), device='cuda')
  da, _ = _with_order('0', lambda: E.pde_values_bwd(Xs, Ys, Lb.PAIRS_FULL, 1,
                                                    Lb.STATIC_RBF, 0.8, g))
  db, _ = _with_order('1', lambda: E.pde_values_bwd(Xs, Ys, Lb.PAIRS_FULL, 1,
                                                    Lb.STATIC_RBF, 0.8, g))
  assert (da - db).abs().max().item() <= 1e-5 * da.abs().max().item()


def test_ragged_form_matches_list_and_differentiates():
  import ksig_b200 as K
  rng = np.random.default_rng(5)
  X, lx = _ragged(rng, 5, 4, 30, 2, torch.float64)
  Y, ly = _ragged(rng, 4, 4, 30, 2, torch.float64)
  kern = K.SignatureKernel(n_levels=3, order=2, static_kernel=K.RBFKernel(1.1))
  xl = [X[i, :lx[i]].detach().clone().requires_grad_(True) for i in range(5)]
  yl = [Y[i, :ly[i]] for i in range(4)]
  k_list = kern(xl, yl, return_on_gpu=True)
  Xg = X.detach().clone().requires_grad_(True)
  k_rag = kern(K.Ragged(Xg, lx), K.Ragged(Y, ly), return_on_gpu=True)
  assert torch.allclose(k_list, k_rag, rtol=1e-12, atol=0)
  W = torch.tensor(rng.standard_normal((5, 4)), device='cuda')
  (k_list * W).sum().backward()
  (k_rag * W).sum().backward()
  for i in range(5):
    assert torch.allclose(xl[i].grad, Xg.grad[i, :lx[i]], rtol=1e-10, atol=1e-14)
    assert float(Xg.grad[i, lx[i]:].abs().max() if lx[i] < X.shape[1] else 0) == 0.0


@pytest.mark.parametrize('pde', [False, True])
def test_graphed_call_replays_eager_result(pde):
  import ksig_b200 as K
  rng = np.random.default_rng(7)
  X, lx = _ragged(rng, 12, 5, 60, 3)
  Y, ly = _ragged(rng, 9, 5, 60, 3)
  kern = (K.SignaturePDEKernel(dyadic_order=1, static_kernel=K.RBFKernel(0.9)) if pde else
          K.SignatureKernel(n_levels=4, order=1, static_kernel=K.RBFKernel(0.9)))
  g = K.GraphedKernel(kern, K.Ragged(X, lx), K.Ragged(Y, ly))
  ref = kern(K.Ragged(X, lx), K.Ragged(Y, ly), return_on_gpu=True)
  out = g()
  assert torch.equal(out, ref)
  X2, lx2 = _ragged(rng, 12, 5, 60, 3)
  ref2 = kern(K.Ragged(X2, lx2), K.Ragged(Y, ly), return_on_gpu=True)
  out2 = g(K.Ragged(X2, lx2))
  assert torch.equal(out2, ref2)


def test_autotune_picks_a_width_and_keeps_results():
  import ksig_b200 as K
  from ksig_b200 import tuning
  rng = np.random.default_rng(9)
  X, lx = _ragged(rng, 16, 20, 300, 3)
  Y, ly = _ragged(rng, 16, 20, 300, 3)
  kern = K.SignatureKernel(n_levels=4, order=1, static_kernel=K.RBFKernel(1.0))
  ref = kern(K.Ragged(X, lx), K.Ragged(Y, ly), return_on_gpu=True)
  try:
    res = tuning.autotune(kern, K.Ragged(X, lx), K.Ragged(Y, ly), backward=True, reps=1)
    assert tuning.OP_DP_FWD in res and tuning.OP_DP_BWD in res
    assert tuning.get_cols(tuning.OP_DP_FWD) == res[tuning.OP_DP_FWD][0]
    out = kern(K.Ragged(X, lx), K.Ragged(Y, ly), return_on_gpu=True)
    assert torch.allclose(out, ref, rtol=2e-5, atol=1e-7)
  finally:
    tuning.reset()
  assert tuning.get_cols(tuning.OP_DP_FWD) == 0


def test_device_status_reaches_python():
  """A length beyond the padded extent is clamped on the device and flagged
  in the workspace status word; the Python layer raises it at the next
  check instead of returning silently."""
  import ksig_b200 as K
  from ksig_b200 import _engine as E, _lib as Lb
  K.check_device_status()  # clean slate
  X = torch.randn((3, 10, 2), device='cuda')
  bad = E.Seqs(X, torch.tensor([10, 12, 5], dtype=torch.int32, device='cuda'))
  E.sig_levels(bad, None, Lb.PAIRS_UPPER, 3, 1, True, Lb.STATIC_RBF, 1.0)
  with pytest.raises(ValueError):
    K.check_device_status()
  K.check_device_status()  # cleared by the raise
  good = E.Seqs(X, torch.tensor([10, 7, 5], dtype=torch.int32, device='cuda'))
  E.sig_levels(good, None, Lb.PAIRS_UPPER, 3, 1, True, Lb.STATIC_RBF, 1.0)
  K.check_device_status()


@pytest.mark.parametrize('batch_size', [None, 4, 7])
def test_precompute_kernel_mat_matches_full_call(batch_size):
  """Block-row precompute (the SVC caller, ksig/models/pre_base.py:88-142)
  equals the single call, for K(X) (mirrored) and K(X, X2)."""
  import ksig_b200 as K
  rng = np.random.default_rng(11)
  X = np.cumsum(rng.standard_normal((13, 20, 3)) * 0.3, axis=1)
  X2 = np.cumsum(rng.standard_normal((6, 15, 3)) * 0.3, axis=1)
  kern = K.SignatureKernel(n_levels=4, order=1, normalize=True,
                           static_kernel=K.RBFKernel(0.8))
  full = kern(X)
  full2 = kern(X, X2)
  got = K.precompute.precompute_kernel_mat(kern, X, None, batch_size)
  got2 = K.precompute.precompute_kernel_mat(kern, X, X2, batch_size)
  assert got.shape == (13, 13) and got2.shape == (13, 6)
  np.testing.assert_allclose(got, full, rtol=1e-12, atol=1e-14)
  np.testing.assert_allclose(got2, full2, rtol=1e-12, atol=1e-14)
  np.testing.assert_allclose(got, got.T, rtol=0, atol=0)


@pytest.mark.parametrize('pde', [False, True])
def test_sharded_sym_gram_single_rank_equals_call(pde):
  """The upper-triangle pair-list path (KSIG_PAIRS_LIST + normalisation of
  the gathered triangle) reproduces K(X); with one rank it is the whole
  triangle."""
  import ksig_b200 as K
  from ksig_b200.distributed import sharded_sym_gram
  rng = np.random.default_rng(31)
  xs = [np.cumsum(rng.standard_normal((n, 3)) * 0.3, 0) for n in (9, 30, 4, 17, 22, 2)]
  kern = (K.SignaturePDEKernel(dyadic_order=1, static_kernel=K.RBFKernel(0.8)) if pde
          else K.SignatureKernel(n_levels=4, order=2, static_kernel=K.RBFKernel(0.8)))
  got = sharded_sym_gram(kern, xs).cpu().numpy()
  np.testing.assert_allclose(got, kern(xs), rtol=1e-12, atol=1e-14)
