"""Pair-grid sharding of a signature Gram across torch.distributed ranks.

Every (x, y) pair of a Gram is independent, so the grid shards with no data
exchange: rank r computes the contiguous row block ``X[rows_r]`` against all
of Y (weak scaling when every rank holds its own block, strong scaling when
one Gram is split).  ``all_gather`` is the only collective, and only when
the caller asks for the assembled matrix.  Normalisation stays exact: a row
block evaluated as ``K(X[rows], Y)`` normalises by the diagonals of both
sides, exactly as the full ``K(X, Y)`` would (ksig/kernels.py:190-214).

Gradients: when the block requires grad, the gather is the differentiable
``torch.distributed.nn`` all-gather, whose backward sums the upstream
gradients of every rank into the block's owner.  A rank's backward then
yields dX for its own rows of X and its partial dY (the contribution of
its block); :func:`allreduce_grads` sums both over the ranks, the one
exchange step the adjoint has.  If every rank evaluates the same loss on
the gathered matrix, scale that loss by 1 / world_size.
"""

from typing import Callable, Optional, Tuple

import torch
import torch.distributed as dist


def shard_rows(n: int, world: int, rank: int) -> Tuple[int, int]:
  """Contiguous row block [start, stop) of rank ``rank`` out of ``world``;
  sizes differ by at most one and cover 0..n-1 exactly once."""
  if world <= 0 or not 0 <= rank < world:
    raise ValueError(f'bad rank {rank} of {world}')
  base, extra = divmod(n, world)
  start = rank * base + min(rank, extra)
  stop = start + base + (1 if rank < extra else 0)
  return start, stop


def sharded_gram(kernel: Callable, X, Y=None, gather: bool = True,
                 group: Optional['dist.ProcessGroup'] = None):
  """Evaluates ``kernel(X, Y)`` with the rows split over the ranks of
  ``group``.

  ``kernel`` is any callable ``(X_block, Y) -> [rows, nY]`` array; for a
  ``ksig_b200`` signature kernel pass ``lambda a, b: K(a, b,
  return_on_gpu=True)``.  ``Y=None`` means K(X): each rank evaluates
  ``kernel(X[rows], X)``.  Returns this rank's block, or with ``gather`` the
  full ``[nX, nY]`` matrix on every rank.
  """
  world = dist.get_world_size(group) if dist.is_initialized() else 1
  rank = dist.get_rank(group) if dist.is_initialized() else 0
  n = len(X)
  start, stop = shard_rows(n, world, rank)
  Yv = X if Y is None else Y
  block = kernel(X[start:stop], Yv)
  block = torch.as_tensor(block)
  if not gather or world == 1:
    return block
  ny = block.shape[1]
  sizes = [shard_rows(n, world, r) for r in range(world)]
  maxrows = max(b - a for a, b in sizes)
  if block.requires_grad:
    import torch.distributed.nn.functional as dnn
    pad = block.new_zeros((maxrows - block.shape[0], ny))
    parts = dnn.all_gather(torch.cat([block, pad], dim=0), group=group)
  else:
    padded = torch.zeros((maxrows, ny), dtype=block.dtype, device=block.device)
    padded[:block.shape[0]] = block
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
  return torch.cat([p[:b - a] for p, (a, b) in zip(parts, sizes)], dim=0)


def allreduce_grads(tensors, group: Optional['dist.ProcessGroup'] = None):
  """Sums ``t.grad`` over the ranks for every tensor that has one (after a
  backward through :func:`sharded_gram`: dX rows live on their owners, dY
  is split into per-rank partial sums)."""
  if not dist.is_initialized():
    return
  for t in tensors:
    if t is not None and t.grad is not None:
      dist.all_reduce(t.grad, op=dist.ReduceOp.SUM, group=group)
