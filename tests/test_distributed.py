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
