"""Multi-rank host logic (gloo, world_size 2, CPU): row sharding of the pair
grid and assembly of the Gram.  The per-block evaluation is the FP64 oracle
standing in for the CUDA kernel, which needs a GPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ksig_b200.distributed import shard_rows


def test_shard_rows_cover_exactly_once():
  for n in (0, 1, 5, 17, 512):
    for world in (1, 2, 3, 8):
      seen = []
      for r in range(world):
        a, b = shard_rows(n, world, r)
        assert 0 <= a <= b <= n
        seen.extend(range(a, b))
      assert seen == list(range(n))
  with pytest.raises(ValueError):
    shard_rows(4, 2, 2)


def _free_port():
  s = socket.socket()
  s.bind(('127.0.0.1', 0))
  p = s.getsockname()[1]
  s.close()
  return p


def _worker(rank, world, port, X, Y, out_q):
  import sys
  sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
  from oracle import ksig_oracle as O
  from ksig_b200.distributed import sharded_gram
  os.environ['MASTER_ADDR'] = '127.0.0.1'
  os.environ['MASTER_PORT'] = str(port)
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    kern = lambda a, b: torch.as_tensor(O.signature_kernel(  # noqa: E731
        np.asarray(a), np.asarray(b), n_levels=3, normalize=True, param=0.7))
    full = sharded_gram(kern, X, Y, gather=True)
    sym = sharded_gram(kern, X, None, gather=True)
    out_q.put((rank, full.numpy(), sym.numpy()))
  finally:
    dist.destroy_process_group()


def test_sharded_gram_two_ranks_gloo():
  rng = np.random.default_rng(0)
  X = np.cumsum(rng.standard_normal((5, 9, 2)) * 0.3, axis=1)
  Y = np.cumsum(rng.standard_normal((3, 7, 2)) * 0.3, axis=1)
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, 2, port, X, Y, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = [q.get(timeout=120) for _ in procs]
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  from oracle import ksig_oracle as O
  ref = O.signature_kernel(X, Y, n_levels=3, normalize=True, param=0.7)
  refx = O.signature_kernel(X, None, n_levels=3, normalize=True, param=0.7)
  for _, full, sym in res:
    np.testing.assert_allclose(full, ref, rtol=1e-12)
    np.testing.assert_allclose(sym, refx, rtol=1e-12)


def _grad_worker(rank, world, port, X, Y, W, out_q):
  import sys
  sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
  from oracle import ksig_oracle_torch as OT
  from ksig_b200.distributed import allreduce_grads, sharded_gram
  os.environ['MASTER_ADDR'] = '127.0.0.1'
  os.environ['MASTER_PORT'] = str(port)
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    Xt = torch.tensor(X, requires_grad=True)
    Yt = torch.tensor(Y, requires_grad=True)

    def kern(a, b):
      return OT.signature_kernel(list(a), list(b), n_levels=3, normalize=True, param=0.7)

    full = sharded_gram(kern, Xt, Yt, gather=True)
    ((full * torch.tensor(W)).sum() / world).backward()
    allreduce_grads([Xt, Yt])
    out_q.put((rank, full.detach().numpy(), Xt.grad.numpy(), Yt.grad.numpy()))
  finally:
    dist.destroy_process_group()


def test_sharded_gram_gradients_two_ranks_gloo():
  """The differentiable gather plus the gradient all-reduce give every rank
  the unsharded dX and dY."""
  from oracle import ksig_oracle_torch as OT
  rng = np.random.default_rng(1)
  X = np.cumsum(rng.standard_normal((5, 7, 2)) * 0.3, axis=1)
  Y = np.cumsum(rng.standard_normal((3, 6, 2)) * 0.3, axis=1)
  W = rng.standard_normal((5, 3))
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_grad_worker, args=(r, 2, port, X, Y, W, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = [q.get(timeout=180) for _ in procs]
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  Xt = torch.tensor(X, requires_grad=True)
  Yt = torch.tensor(Y, requires_grad=True)
  ref = OT.signature_kernel(list(Xt), list(Yt), n_levels=3, normalize=True, param=0.7)
  (ref * torch.tensor(W)).sum().backward()
  for _, full, gx, gy in res:
    np.testing.assert_allclose(full, ref.detach().numpy(), rtol=1e-12)
    np.testing.assert_allclose(gx, Xt.grad.numpy(), rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(gy, Yt.grad.numpy(), rtol=1e-10, atol=1e-14)


def test_split_by_cost_balances_and_covers():
  from ksig_b200.distributed import split_by_cost, upper_pairs
  p = upper_pairs(5)
  assert p.shape == (15, 2) and (p[:, 0] <= p[:, 1]).all()
  assert p[:5].tolist() == [[0, 0], [0, 1], [0, 2], [0, 3], [0, 4]]
  cost = np.r_[np.ones(10), np.full(10, 9.0)]
  b = split_by_cost(cost, 4)
  assert b[0] == 0 and b[-1] == 20 and (np.diff(b) >= 0).all()
  sums = [cost[b[r]:b[r + 1]].sum() for r in range(4)]
  assert max(sums) - min(sums) <= 9.0


def _sym_worker(rank, world, port, xs, out_q):
  import sys
  sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
  from oracle import ksig_oracle as O
  from ksig_b200.distributed import sharded_sym_levels
  os.environ['MASTER_ADDR'] = '127.0.0.1'
  os.environ['MASTER_PORT'] = str(port)
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    def levels_fn(pairs):
      # One pair at a time through the oracle: [n_levels + 1, len(pairs)].
      cols = [O.signature_kernel([xs[a]], [xs[b]], n_levels=3, return_levels=True,
                                 param=0.7)[:, 0, 0] for a, b in pairs]
      return torch.tensor(np.stack(cols, axis=1)) if cols else torch.zeros((4, 0), dtype=torch.float64)
    lev = sharded_sym_levels(levels_fn, [len(x) for x in xs])
    out_q.put((rank, lev.numpy()))
  finally:
    dist.destroy_process_group()


def test_sharded_sym_levels_two_ranks_gloo():
  """The cost-balanced upper-triangle split plus one all_gather gives every
  rank the full per-level array in KSIG_PAIRS_UPPER order."""
  from oracle import ksig_oracle as O
  from ksig_b200.distributed import upper_pairs
  rng = np.random.default_rng(2)
  xs = [np.cumsum(rng.standard_normal((n, 2)) * 0.3, 0) for n in (4, 15, 7, 11, 3)]
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_sym_worker, args=(r, 2, port, xs, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = [q.get(timeout=180) for _ in procs]
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  full = O.signature_kernel(xs, None, n_levels=3, return_levels=True, param=0.7)
  pairs = upper_pairs(len(xs))
  ref = full[:, pairs[:, 0], pairs[:, 1]]
  for _, lev in res:
    np.testing.assert_allclose(lev, ref, rtol=1e-12, atol=1e-14)
