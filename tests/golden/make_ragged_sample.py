"""Oracle values for the sample that bench.py checks on the ragged workload.

The ragged order-2 workload of ``bench.py`` (N = M = 2048 sequences, lengths
log-uniform in [32, 1024], d = 16 cumsummed N(0, 1) increments, RBF bandwidth
4, n_levels = 8, order = 2, normalised) is generated from seeded NumPy
streams (``bench.make_ragged``, seeds 5 and 6).  This script picks a sample
of it that holds the longest sequences of each side, evaluates the FP64
oracle on the FP32-rounded inputs and writes ``ragged_dp_sample.npz``:

  ix, iy   sequence indices of the sample (4 + 4)
  K        normalised K(X_s, Y_s), [4, 4] float64
  gx, gy   indices of the gradient sample (2 + 2; a sub-sample of ix, iy)
  W        weights of L = sum(W * K(X_g, Y_g)), [2, 2]
  dX       dL/dX_g through autograd of the FP64 torch oracle, [2, Lmax, 16]
           (zero past each sequence's length)

so that the bench reports per-entry errors against the oracle without
running it.  Run from the repository root:

    python tests/golden/make_ragged_sample.py
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle import ksig_oracle as O  # noqa: E402
from oracle import ksig_oracle_torch as OT  # noqa: E402


def sample_indices(X, Y):
  """Two longest and two median-length sequences of each side."""
  def pick(S):
    lens = np.array([s.shape[0] for s in S])
    order = np.argsort(-lens, kind='stable')
    return np.array([order[0], order[1], order[len(S) // 2], order[len(S) // 2 + 1]])
  return pick(X), pick(Y)


def main():
  R = bench.RAGGED
  X = bench.make_ragged(R['n'], R['lmin'], R['lmax'], R['d'], 5)
  Y = bench.make_ragged(R['n'], R['lmin'], R['lmax'], R['d'], 6)
  ix, iy = sample_indices(X, Y)
  Xs = [X[i].astype(np.float64) for i in ix]
  Ys = [Y[i].astype(np.float64) for i in iy]
  K = O.signature_kernel(Xs, Ys, n_levels=R['n_levels'], order=R['order'],
                         normalize=True, param=R['bw'])
  gx, gy = ix[:2], iy[:2]
  W = np.random.default_rng(17).standard_normal((2, 2))
  Xo = [torch.tensor(X[i].astype(np.float64), requires_grad=True) for i in gx]
  Yo = [torch.tensor(Y[i].astype(np.float64)) for i in gy]
  ref = OT.signature_kernel(Xo, Yo, n_levels=R['n_levels'], order=R['order'],
                            normalize=True, param=R['bw'])
  (ref * torch.tensor(W)).sum().backward()
  Lm = max(x.shape[0] for x in Xo)
  dX = np.zeros((2, Lm, R['d']))
  for j, x in enumerate(Xo):
    dX[j, :x.shape[0]] = x.grad.numpy()
  path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'ragged_dp_sample.npz')
  np.savez_compressed(path, ix=ix, iy=iy, K=K, gx=gx, gy=gy, W=W, dX=dX)
  print('wrote', path, 'lengths', [X[i].shape[0] for i in ix], [Y[i].shape[0] for i in iy])


if __name__ == '__main__':
  main()
