"""Reader for ``tests/golden/golden.npz`` (reference outputs + inputs)."""
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden',
                    'golden.npz')


def load_cases():
  z = np.load(PATH)
  meta = json.loads(str(z['__meta__']))
  cases = []
  for m in meta:
    n = m['name']
    if m['ragged']:
      X = [z[f'{n}/X{i}'] for i in range(m['nx'])]
      Y = [z[f'{n}/Y{i}'] for i in range(m['ny'])]
    else:
      X, Y = z[f'{n}/X'], z[f'{n}/Y']
    cases.append(dict(m, X=X, Y=Y, KXX=z[f'{n}/KXX'], KXY=z[f'{n}/KXY'],
                      Kdiag=z[f'{n}/Kdiag']))
  return cases
