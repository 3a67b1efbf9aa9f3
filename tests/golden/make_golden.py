"""Generates the golden fixtures in this folder from the reference KSig itself.

Run from the repository root, in a container that has the reference source
checked out at ``--ref`` (a path to the KSig 1.0.0 source tree)::

    python tests/golden/make_golden.py --ref <path to the KSig source tree>

The reference needs CuPy and a CUDA device.  Neither is needed here: the
NumPy-backed ``cupy`` stand-in in ``tests/_refshim`` takes CuPy's place and
Numba's CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``) runs the Numba PDE and
global-alignment kernels of ksig/algorithms.py unchanged.  Every case stores
its inputs, its parameters and the reference's outputs in ``golden.npz``
(kernels) and ``preprocessing.npz`` (ksig/preprocessing.py); the tests read
only those files, never the reference.
"""

import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(os.path.dirname(HERE), '_refshim')


def _cases():
  import numpy as np
  cases = []

  def add(name, kernel, params, X, Y=None, ragged=False):
    cases.append(dict(name=name, kernel=kernel, params=params, X=X, Y=Y,
                      ragged=ragged))

  rng = np.random.default_rng(0)
  X0 = rng.standard_normal((10, 50, 5))
  Y0 = rng.standard_normal((8, 20, 5))
  base = dict(n_levels=5, order=1, normalize=False, static='rbf', param=1.0)
  add('cfg1_dp_rbf', 'sig', base, X0, Y0)
  add('cfg1_dp_rbf_norm', 'sig', dict(base, normalize=True), X0, Y0)

  rng = np.random.default_rng(10)
  X1 = np.cumsum(rng.standard_normal((6, 17, 3)) * 0.3, axis=1)
  Y1 = np.cumsum(rng.standard_normal((5, 13, 3)) * 0.3, axis=1)
  add('dp_o2_m4', 'sig', dict(n_levels=4, order=2, normalize=False,
                               static='rbf', param=0.7), X1, Y1)
  add('dp_o2_m4_norm', 'sig', dict(n_levels=4, order=2, normalize=True,
                                    static='rbf', param=0.7), X1, Y1)
  add('dp_o3_m5', 'sig', dict(n_levels=5, order=3, normalize=False,
                               static='rbf', param=1.3), X1, Y1)
  add('dp_ofull_m3', 'sig', dict(n_levels=3, order=0, normalize=False,
                                  static='rbf', param=1.0), X1, Y1)
  add('dp_linear', 'sig', dict(n_levels=4, order=1, normalize=False,
                                static='linear', param=0.5), X1, Y1)
  add('dp_linear_norm', 'sig', dict(n_levels=4, order=1, normalize=True,
                                     static='linear', param=0.5), X1, Y1)
  add('dp_nodiff', 'sig', dict(n_levels=3, order=1, normalize=False,
                                difference=False, static='rbf', param=2.0),
      X1[:, :9], Y1[:, :7])
  add('dp_m1', 'sig', dict(n_levels=1, order=1, normalize=True,
                            static='rbf', param=1.0), X1, Y1)
  rng = np.random.default_rng(11)
  add('dp_d1_L2', 'sig', dict(n_levels=3, order=1, normalize=False,
                               static='rbf', param=1.0),
      rng.standard_normal((4, 2, 1)), rng.standard_normal((3, 2, 1)))
  add('dp_L1', 'sig', dict(n_levels=3, order=1, normalize=False,
                            static='rbf', param=1.0),
      rng.standard_normal((3, 1, 2)), rng.standard_normal((2, 5, 2)))

  # Ragged batch pinned through the reference's padding invariance: the
  # reference sees edge-padded dense arrays, the fixture keeps the lengths.
  rng = np.random.default_rng(12)
  lens_x = [7, 12, 3, 9]
  lens_y = [5, 12, 10]
  xs = [np.cumsum(rng.standard_normal((n, 2)) * 0.4, axis=0) for n in lens_x]
  ys = [np.cumsum(rng.standard_normal((n, 2)) * 0.4, axis=0) for n in lens_y]
  add('dp_ragged_o1', 'sig', dict(n_levels=4, order=1, normalize=True,
                                   static='rbf', param=0.8), xs, ys,
      ragged=True)
  add('dp_ragged_o2', 'sig', dict(n_levels=4, order=2, normalize=False,
                                   static='rbf', param=0.8), xs, ys,
      ragged=True)

  rng = np.random.default_rng(1)
  A = rng.standard_normal((2, 8, 3))
  B = rng.standard_normal((2, 6, 3))
  add('pde_rbf', 'pde', dict(normalize=False, static='rbf', param=1.0), A, B)
  add('pde_rbf_norm', 'pde', dict(normalize=True, static='rbf', param=1.0),
      A, B)
  rng = np.random.default_rng(13)
  P = np.cumsum(rng.standard_normal((3, 9, 2)) * 0.5, axis=1)
  Q = np.cumsum(rng.standard_normal((2, 11, 2)) * 0.5, axis=1)
  add('pde_linear', 'pde', dict(normalize=False, static='linear', param=0.6),
      P, Q)
  add('pde_ragged', 'pde', dict(normalize=False, static='rbf', param=0.9),
      [P[0, :5], P[1], P[2, :7]], [Q[0, :4], Q[1]], ragged=True)

  # The other static kernels of ksig.static.kernels (Matern12 / 32 go
  # through the reference's euclid_dist, which measures within the second
  # point set, so they have no reference output to pin to).
  add('dp_poly', 'sig', dict(n_levels=3, order=1, normalize=False,
                              static='poly', param=[2.0, 1.0, 0.5]),
      X1[:, :9], Y1[:, :7])
  add('dp_poly_o2_norm', 'sig', dict(n_levels=3, order=2, normalize=True,
                                      static='poly', param=[3.0, 0.5, 1.0]),
      X1[:, :9], Y1[:, :7])
  add('dp_matern52', 'sig', dict(n_levels=4, order=1, normalize=False,
                                  static='matern52', param=0.9), X1, Y1)
  add('dp_matern52_norm', 'sig', dict(n_levels=4, order=1, normalize=True,
                                       static='matern52', param=0.9), X1, Y1)
  add('dp_rq', 'sig', dict(n_levels=4, order=2, normalize=False,
                            static='rq', param=[0.8, 1.5]), X1, Y1)
  add('pde_matern52', 'pde', dict(normalize=False, static='matern52', param=1.1),
      P, Q)
  add('pde_rq_norm', 'pde', dict(normalize=True, static='rq', param=[0.7, 2.0]),
      P, Q)
  add('pde_poly', 'pde', dict(normalize=False, static='poly', param=[2.0, 1.0, 0.3]),
      P[:, :6], Q[:, :5])

  # Full order beyond 4 (order 0 -> order = n_levels, ksig/kernels.py:
  # 49-50), deeper truncations, and more channels than the register-Gram
  # tiles hold (the Gram-input path).
  add('dp_ofull_m6_norm', 'sig', dict(n_levels=6, order=0, normalize=True,
                                       static='rbf', param=0.9), X1, Y1)
  add('dp_o5_m8', 'sig', dict(n_levels=8, order=5, normalize=False,
                               static='rbf', param=1.1), X1[:, :11], Y1[:, :9])
  add('dp_ofull_m10', 'sig', dict(n_levels=10, order=0, normalize=False,
                                   static='rbf', param=1.0), X1[:3, :8], Y1[:2, :7])
  add('dp_m16_norm', 'sig', dict(n_levels=16, order=1, normalize=True,
                                  static='rbf', param=0.8), X1, Y1)
  add('dp_o2_m12', 'sig', dict(n_levels=12, order=2, normalize=False,
                                static='rbf', param=0.8), X1, Y1)
  rng = np.random.default_rng(15)
  W1 = np.cumsum(rng.standard_normal((4, 23, 64)) * 0.2, axis=1)
  W2 = np.cumsum(rng.standard_normal((3, 19, 64)) * 0.2, axis=1)
  add('dp_d64_norm', 'sig', dict(n_levels=4, order=1, normalize=True,
                                  static='rbf', param=2.0), W1, W2)
  add('dp_d64_o2', 'sig', dict(n_levels=4, order=2, normalize=False,
                                static='rbf', param=2.0), W1, W2)
  add('dp_d40_linear', 'sig', dict(n_levels=3, order=1, normalize=True,
                                    static='linear', param=0.3),
      W1[:, :, :40], W2[:, :, :40])
  add('dp_d40_matern52', 'sig', dict(n_levels=4, order=1, normalize=False,
                                      static='matern52', param=2.5),
      W1[:, :, :40], W2[:, :, :40])
  add('dp_d64_ragged', 'sig', dict(n_levels=4, order=1, normalize=True,
                                    static='rbf', param=2.0),
      [W1[0, :9], W1[1], W1[2, :15]], [W2[0, :4], W2[1], W2[2, :12]], ragged=True)
  add('pde_d48_norm', 'pde', dict(normalize=True, static='rbf', param=2.0),
      W1[:, :, :48], W2[:, :, :48])

  # Global alignment kernel (ksig/kernels.py:366-409).
  rng = np.random.default_rng(14)
  G1 = np.cumsum(rng.standard_normal((4, 11, 3)) * 0.4, axis=1)
  G2 = np.cumsum(rng.standard_normal((3, 8, 3)) * 0.4, axis=1)
  add('ga_rbf', 'ga', dict(normalize=True, static='rbf', param=1.2), G1, G2)
  add('ga_linear', 'ga', dict(normalize=True, static='linear', param=0.4), G1, G2)
  add('ga_d40', 'ga', dict(normalize=True, static='rbf', param=3.0),
      W1[:, :11, :40], W2[:, :8, :40])
  return cases


def _static(ksig, p):
  st, v = p['static'], p['param']
  K = ksig.static.kernels
  if st == 'rbf':
    return K.RBFKernel(v)
  if st == 'linear':
    return K.LinearKernel(v)
  if st == 'poly':
    return K.PolynomialKernel(degree=v[0], gamma=v[1], scale=v[2])
  if st == 'matern52':
    return K.Matern52Kernel(v)
  if st == 'rq':
    return K.RationalQuadraticKernel(bandwidth=v[0], alpha=v[1])
  raise ValueError(st)


def _pad_edge(seqs):
  import numpy as np
  L = max(s.shape[0] for s in seqs)
  return np.stack([np.concatenate([s, np.repeat(s[-1:], L - len(s), 0)], 0)
                   for s in seqs])


def _run_reference():
  """Runs inside the shimmed interpreter; returns nothing, writes npz."""
  import numba.cuda
  numba.cuda.default_stream = lambda: 0
  import numpy as np
  import ksig
  out = {}
  meta = []
  for c in _cases():
    p = c['params']
    static = _static(ksig, p)
    if c['kernel'] == 'sig':
      K = ksig.kernels.SignatureKernel(
          n_levels=p['n_levels'], order=p['order'],
          difference=p.get('difference', True), normalize=p['normalize'],
          static_kernel=static)
    elif c['kernel'] == 'pde':
      K = ksig.kernels.SignaturePDEKernel(
          difference=p.get('difference', True), normalize=p['normalize'],
          static_kernel=static)
    else:
      K = ksig.kernels.GlobalAlignmentKernel(static_kernel=static)
    X, Y = c['X'], c['Y']
    name = c['name']
    if c['ragged']:
      for i, s in enumerate(X):
        out[f'{name}/X{i}'] = s
      for i, s in enumerate(Y):
        out[f'{name}/Y{i}'] = s
      Xd, Yd = _pad_edge(X), _pad_edge(Y)
      nx, ny = len(X), len(Y)
    else:
      out[f'{name}/X'] = X
      out[f'{name}/Y'] = Y
      Xd, Yd = X, Y
      nx, ny = X.shape[0], Y.shape[0]
    out[f'{name}/KXX'] = np.asarray(K(Xd))
    out[f'{name}/KXY'] = np.asarray(K(Xd, Yd))
    out[f'{name}/Kdiag'] = np.asarray(K(Xd, diag=True), dtype=np.float64)
    meta.append(dict(name=name, kernel=c['kernel'], params=p,
                     ragged=c['ragged'], nx=nx, ny=ny))
  out['__meta__'] = np.array(json.dumps(meta))
  np.savez_compressed(os.path.join(HERE, 'golden.npz'), **out)
  print('wrote', len(meta), 'cases')


def _run_preprocessing():
  """Reference outputs of ksig/preprocessing.py (writes preprocessing.npz)."""
  import numpy as np
  import ksig
  P = ksig.preprocessing
  rng = np.random.default_rng(21)
  out = {}
  seqs = [np.cumsum(rng.standard_normal((n, 2)), 0) for n in (5, 9, 7)]
  seqs[1][3, 1] = np.nan
  for i, s in enumerate(seqs):
    out[f'tab_ragged/in{i}'] = s
  out['tab_ragged/out'] = P.SequenceTabulator().fit(seqs).transform(seqs)
  eq = rng.standard_normal((3, 8, 2))
  out['tab_max6/in'] = eq
  out['tab_max6/out'] = P.SequenceTabulator(max_len=6).fit(eq).transform(eq.copy())
  out['tab_same/in'] = eq
  out['tab_same/out'] = P.SequenceTabulator().fit(eq).transform(eq.copy())
  X = np.abs(rng.standard_normal((3, 10, 2))) + 0.5
  out['aug_default/in'] = X
  out['aug_default/out'] = P.SequenceAugmentor().fit(X).transform(X.copy())
  A = P.SequenceAugmentor(lead_lag=False, max_time=2.5, basepoint=False,
                          normalize=False)
  out['aug_time/in'] = X
  out['aug_time/out'] = A.fit(X).transform(X.copy())
  out['aug_maxlen/in'] = X
  out['aug_maxlen/out'] = P.SequenceAugmentor(max_len=15).fit(X).transform(X.copy())
  np.savez_compressed(os.path.join(HERE, 'preprocessing.npz'), **out)
  print('wrote preprocessing fixtures')


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--ref', required=True,
                  help='KSig 1.0.0 source tree (the directory holding ksig/)')
  ap.add_argument('--_child', action='store_true')
  a = ap.parse_args()
  if a._child:
    _run_reference()
    _run_preprocessing()
    return
  env = dict(os.environ)
  env['PYTHONPATH'] = os.pathsep.join([SHIM, a.ref])
  env['NUMBA_ENABLE_CUDASIM'] = '1'
  subprocess.run([sys.executable, '-W', 'ignore', os.path.abspath(__file__),
                  '--ref', a.ref, '--_child'], env=env, check=True, cwd='/tmp')


if __name__ == '__main__':
  main()
