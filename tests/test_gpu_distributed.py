"""The sharded Gram paths with the CUDA kernels on two ranks.

Two processes share cuda:0 over a gloo process group: each rank runs its own
shard through the library's kernels (no kernel waits on another rank), and the
collectives (all_gather, the differentiable all_gather, the gradient
all-reduce) run through gloo.  Results must equal the single-process calls:
sharded K(X) over the cost-balanced upper triangle (DP and PDE), row-sharded
K(X, Y), and dX / dY after allreduce_grads.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
  s = socket.socket()
  s.bind(('127.0.0.1', 0))
  p = s.getsockname()[1]
  s.close()
  return p


def _data():
  rng = np.random.default_rng(3)
  xs = [np.cumsum(rng.standard_normal((n, 3)) * 0.3, 0).astype(np.float64)
        for n in (9, 30, 4, 17, 22, 2, 26)]
  X = np.cumsum(rng.standard_normal((5, 12, 3)) * 0.3, axis=1)
  Y = np.cumsum(rng.standard_normal((4, 10, 3)) * 0.3, axis=1)
  W = rng.standard_normal((5, 4))
  return xs, X, Y, W


def _worker(rank, world, port, out_q):
  import sys
  sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
  import datetime
  os.environ['MASTER_ADDR'] = '127.0.0.1'
  os.environ['MASTER_PORT'] = str(port)
  torch.cuda.set_device(0)
  dist.init_process_group('gloo', rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=120))
  try:
    import ksig_b200 as K
    from ksig_b200.distributed import allreduce_grads, sharded_gram, sharded_sym_gram
    xs, X, Y, W = _data()
    dp = K.SignatureKernel(n_levels=4, order=2, static_kernel=K.RBFKernel(0.8))
    pde = K.SignaturePDEKernel(dyadic_order=1, static_kernel=K.RBFKernel(0.8))
    sym_dp = sharded_sym_gram(dp, xs).cpu().numpy()
    sym_pde = sharded_sym_gram(pde, xs).cpu().numpy()
    Xt = torch.tensor(X, device='cuda', requires_grad=True)
    Yt = torch.tensor(Y, device='cuda', requires_grad=True)
    k1 = K.SignatureKernel(n_levels=4, order=1, static_kernel=K.RBFKernel(0.7))
    full = sharded_gram(lambda a, b: k1(a, b, return_on_gpu=True).cpu(), Xt, Yt, gather=True)
    ((full * torch.tensor(W)).sum() / world).backward()
    allreduce_grads([Xt, Yt])
    out_q.put((rank, sym_dp, sym_pde, full.detach().numpy(), Xt.grad.cpu().numpy(),
               Yt.grad.cpu().numpy()))
  finally:
    dist.destroy_process_group()


def test_sharded_paths_two_ranks_cuda_kernels():
  import ksig_b200 as K
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = [q.get(timeout=300) for _ in procs]
  for p in procs:
    p.join(timeout=120)
    assert p.exitcode == 0
  xs, X, Y, W = _data()
  dp = K.SignatureKernel(n_levels=4, order=2, static_kernel=K.RBFKernel(0.8))
  pde = K.SignaturePDEKernel(dyadic_order=1, static_kernel=K.RBFKernel(0.8))
  ref_dp, ref_pde = dp(xs), pde(xs)
  Xt = torch.tensor(X, device='cuda', requires_grad=True)
  Yt = torch.tensor(Y, device='cuda', requires_grad=True)
  k1 = K.SignatureKernel(n_levels=4, order=1, static_kernel=K.RBFKernel(0.7))
  ref = k1(Xt, Yt, return_on_gpu=True)
  (ref * torch.tensor(W, device='cuda')).sum().backward()
  for _, sdp, spde, full, gx, gy in res:
    np.testing.assert_allclose(sdp, ref_dp, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(spde, ref_pde, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(full, ref.detach().cpu().numpy(), rtol=1e-12)
    np.testing.assert_allclose(gx, Xt.grad.cpu().numpy(), rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(gy, Yt.grad.cpu().numpy(), rtol=1e-9, atol=1e-13)
