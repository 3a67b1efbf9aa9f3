"""Pins the FP64 oracle against outputs of the reference KSig package."""
import numpy as np
import pytest

from golden_io import load_cases
from oracle import ksig_oracle as O

CASES = load_cases()


def _oracle(c, X, Y=None, diag=False):
  p = c['params']
  if c['kernel'] == 'sig':
    return O.signature_kernel(
        X, Y, diag=diag, n_levels=p['n_levels'], order=p['order'],
        difference=p.get('difference', True), normalize=p['normalize'],
        kind=p['static'], param=p['param'])
  if c['kernel'] == 'ga':
    return O.global_align_kernel(X, Y, diag=diag, kind=p['static'], param=p['param'])
  return O.signature_pde_kernel(
      X, Y, diag=diag, difference=p.get('difference', True),
      normalize=p['normalize'], kind=p['static'], param=p['param'])


@pytest.mark.parametrize('c', CASES, ids=[c['name'] for c in CASES])
def test_oracle_matches_reference(c):
  np.testing.assert_allclose(_oracle(c, c['X']), c['KXX'], rtol=1e-12,
                             atol=1e-12)
  np.testing.assert_allclose(_oracle(c, c['X'], c['Y']), c['KXY'],
                             rtol=1e-12, atol=1e-12)
  np.testing.assert_allclose(_oracle(c, c['X'], diag=True), c['Kdiag'],
                             rtol=1e-12, atol=1e-12)


def test_survey_golden_values():
  """Literal values of the reference on the 10x50x5 / 8x20x5 seed-0 case."""
  c = [c for c in CASES if c['name'] == 'cfg1_dp_rbf'][0]
  K = c['KXX']
  assert K[0, 0] == pytest.approx(21065.176612755662, rel=1e-14)
  assert K[0, 1] == pytest.approx(176.80966800828605, rel=1e-14)
  assert K[9, 8] == pytest.approx(167.04767717247762, rel=1e-14)
  assert c['KXY'][0, 0] == pytest.approx(34.748845291785315, rel=1e-14)
  assert c['KXY'][9, 7] == pytest.approx(40.31632099023666, rel=1e-14)
  p = [c for c in CASES if c['name'] == 'pde_rbf'][0]
  np.testing.assert_allclose(
      p['KXY'], [[1.3323776075844755, 1.1142179302362047],
                 [1.39303056405124, 0.7423432806317123]], rtol=1e-14)


def test_pde_dyadic_refinement_converges():
  """Dyadic refinement of the Goursat scheme converges (no reference
  counterpart; order 0 is the reference scheme)."""
  rng = np.random.default_rng(5)
  x = np.cumsum(rng.standard_normal((12, 2)) * 0.3, axis=0)
  y = np.cumsum(rng.standard_normal((10, 2)) * 0.3, axis=0)
  Z = O.second_difference(O.static_gram(x, y, 'rbf', 0.5))
  v = [O.sig_pde(Z, k) for k in range(5)]
  d = [abs(v[k + 1] - v[k]) for k in range(4)]
  assert d[3] < d[2] < d[1] < d[0]


def test_padding_invariance_oracle():
  rng = np.random.default_rng(6)
  x = rng.standard_normal((9, 3))
  y = rng.standard_normal((6, 3))
  xp = np.concatenate([x, np.repeat(x[-1:], 5, 0)])
  for fn in (lambda a, b: O.signature_kernel([a], [b], n_levels=4, order=2,
                                             normalize=False),
             lambda a, b: O.signature_pde_kernel([a], [b], normalize=False,
                                                 dyadic_order=1)):
    np.testing.assert_allclose(fn(xp, y), fn(x, y), rtol=1e-12)
