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

from typing import Callable, Optional, Sequence, Tuple

import numpy as np
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


def upper_pairs(n: int) -> np.ndarray:
  """The upper triangle of an n x n Gram (a <= b), row-major: the order of
  the library's KSIG_PAIRS_UPPER enumeration.  int32 [n(n+1)/2, 2]."""
  a, b = np.triu_indices(n)
  return np.stack([a, b], axis=1).astype(np.int32)


def split_by_cost(cost: Sequence[float], world: int) -> np.ndarray:
  """Boundaries [world + 1] of contiguous chunks of ``cost`` with near-equal
  totals (rank r takes items bounds[r]:bounds[r+1])."""
  c = np.cumsum(np.asarray(cost, dtype=np.float64))
  total = c[-1] if len(c) else 0.0
  cuts = [int(np.searchsorted(c, total * r / world, side='left')) for r in range(1, world)]
  return np.array([0] + cuts + [len(c)], dtype=np.int64)


def sharded_sym_levels(levels_fn: Callable, lengths: Sequence[int],
                       group: Optional['dist.ProcessGroup'] = None):
  """Per-level values of K(X) over the upper triangle, sharded by cost.

  The upper-triangle pair list is cut into contiguous chunks of equal cell
  count (``(L_a - 1)(L_b - 1)`` per pair, so ragged batches balance), rank r
  evaluates its chunk with ``levels_fn(pairs) -> [n_levels + 1, len(pairs)]``
  (for a ``ksig_b200`` kernel: the level kernels of an explicit pair list),
  and one all_gather assembles the full ``[n_levels + 1, n(n+1)/2]`` array in
  upper-triangle order on every rank, ready for the normalisation.  Half the
  pairs of the row-block split, and no pair twice.
  """
  world = dist.get_world_size(group) if dist.is_initialized() else 1
  rank = dist.get_rank(group) if dist.is_initialized() else 0
  n = len(lengths)
  pairs = upper_pairs(n)
  lx = np.maximum(np.asarray(lengths, dtype=np.float64) - 1, 1)
  bounds = split_by_cost(lx[pairs[:, 0]] * lx[pairs[:, 1]], world)
  mine = pairs[bounds[rank]:bounds[rank + 1]]
  lev = torch.as_tensor(levels_fn(mine))
  if world == 1:
    return lev
  counts = [int(bounds[r + 1] - bounds[r]) for r in range(world)]
  pad = max(counts)
  buf = lev.new_zeros((lev.shape[0], pad))
  buf[:, :lev.shape[1]] = lev
  parts = [torch.empty_like(buf) for _ in range(world)]
  dist.all_gather(parts, buf, group=group)
  return torch.cat([p[:, :c] for p, c in zip(parts, counts)], dim=1)


def sharded_sym_gram(kernel, X, group: Optional['dist.ProcessGroup'] = None):
  """K(X) of a ``ksig_b200`` SignatureKernel / SignaturePDEKernel with the
  upper triangle sharded over the ranks (see :func:`sharded_sym_levels`);
  returns the normalised ``[n, n]`` matrix on every rank."""
  from . import _engine as E
  from . import _lib as L
  from .kernels import SignaturePDEKernel, _to_seqs
  Xs, _, _ = _to_seqs(X, kernel.n_features)
  lengths = (Xs.lengths.cpu().numpy() if Xs.lengths is not None
             else np.full((Xs.n,), Xs.L))

  def levels_fn(pairs):
    pl = torch.as_tensor(pairs, device=Xs.data.device).contiguous()
    kind, param = kernel._static()
    if isinstance(kernel, SignaturePDEKernel):
      return E.pde_values(Xs, Xs, L.PAIRS_LIST, kernel.dyadic_order, kernel.difference,
                          kind, param, pair_list=pl)[None, :]
    return E.sig_levels(Xs, Xs, L.PAIRS_LIST, kernel.n_levels, kernel.order,
                        kernel.difference, kind, param, pair_list=pl)

  lev = sharded_sym_levels(levels_fn, lengths, group)
  return E.normalize_levels(lev.contiguous(), L.PAIRS_UPPER, Xs.n, Xs.n, None, None,
                            kernel.normalize, Xs.data.dtype)
