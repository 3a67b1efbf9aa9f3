"""Device preprocessing (ksig_b200.preprocessing) against outputs of the
reference's ksig/preprocessing.py (tests/golden/preprocessing.npz, written by
tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden',
                         'preprocessing.npz'))


def test_tabulator_matches_reference():
  from ksig_b200.preprocessing import SequenceTabulator
  seqs = [Z[f'tab_ragged/in{i}'] for i in range(3)]
  got = SequenceTabulator().fit(seqs).transform(seqs)
  np.testing.assert_allclose(got, Z['tab_ragged/out'], rtol=1e-12, atol=1e-12)
  eq = Z['tab_max6/in']
  np.testing.assert_allclose(SequenceTabulator(max_len=6).fit(eq).transform(eq),
                             Z['tab_max6/out'], rtol=1e-12, atol=1e-12)
  np.testing.assert_array_equal(SequenceTabulator().fit(eq).transform(eq), Z['tab_same/out'])


def test_tabulator_ragged_batch_feeds_the_kernels():
  """ragged=True keeps the true lengths (NaN rows dropped) instead of
  interpolating; the signature kernel on it equals the kernel on the list."""
  import ksig_b200 as K
  from ksig_b200.preprocessing import SequenceTabulator
  seqs = [Z[f'tab_ragged/in{i}'] for i in range(3)]
  rb = SequenceTabulator(ragged=True).fit(seqs).transform(seqs)
  assert isinstance(rb, K.Ragged)
  assert rb.lengths.tolist() == [5, 8, 7]
  clean = [s[np.all(~np.isnan(s), axis=-1)] for s in seqs]
  kern = K.SignatureKernel(n_levels=3, static_kernel=K.RBFKernel(1.5))
  np.testing.assert_allclose(kern(rb), kern(clean), rtol=1e-12)


@pytest.mark.parametrize('case,kw', [('aug_default', {}),
                                     ('aug_time', dict(lead_lag=False, max_time=2.5,
                                                       basepoint=False, normalize=False)),
                                     ('aug_maxlen', dict(max_len=15))])
def test_augmentor_matches_reference(case, kw):
  from ksig_b200.preprocessing import SequenceAugmentor
  X = Z[f'{case}/in']
  X0 = X.copy()
  got = SequenceAugmentor(**kw).fit(X).transform(X)
  np.testing.assert_allclose(got, Z[f'{case}/out'], rtol=1e-12, atol=1e-12)
  np.testing.assert_array_equal(X, X0)  # the input is left alone
  t = SequenceAugmentor(**kw).fit(torch.tensor(X, device='cuda')).transform(
      torch.tensor(X, device='cuda'))
  assert t.is_cuda
  np.testing.assert_allclose(t.cpu().numpy(), Z[f'{case}/out'], rtol=1e-12, atol=1e-12)
