"""The C-ABI library loads and exports every entry point of include/*.h."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, 'ksig_b200', 'lib', 'libksig_b200.so')


def _declared():
  names = set()
  for h in glob.glob(os.path.join(ROOT, 'include', '*.h')):
    text = open(h).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    for m in re.finditer(r'\b(ksig_\w+)\s*\(', text):
      names.add(m.group(1))
  return sorted(names)


@pytest.mark.skipif(not os.path.exists(LIB), reason='library not built')
def test_library_exports_all_declared_symbols():
  lib = ctypes.CDLL(LIB)
  declared = _declared()
  assert declared, 'no declarations found'
  missing = [n for n in declared if not hasattr(lib, n)]
  assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason='library not built')
def test_python_binding_covers_declared_symbols():
  from ksig_b200 import _lib
  bound = set(_lib.exported_symbols()) | set(_lib._OPTIONAL)
  assert set(_declared()) <= bound


@pytest.mark.skipif(not os.path.exists(LIB), reason='library not built')
def test_host_checks_without_gpu():
  """Argument validation runs on the host and reports ValueError-class codes."""
  from ksig_b200 import _lib
  lib = _lib.lib()
  assert lib.ksig_version().startswith(b'ksig_b200')
  assert lib.ksig_num_pairs(_lib.PAIRS_UPPER, 4, 0, 0) == 10
  assert lib.ksig_num_pairs(_lib.PAIRS_FULL, 4, 3, 0) == 12
  rc = lib.ksig_signature_kern(None, None, 2, 5, None, None, 2, 5, 3, 0, 0,
                               1.0, 3, 1, 1, 0, None, 0, None, None, 0, None)
  assert rc == _lib.ERR_INVALID
  assert 'X is NULL' in _lib.last_error()
  rc = lib.ksig_signature_kern(ctypes.c_void_p(16), None, 2, 5,
                               ctypes.c_void_p(16), None, 2, 5, 3, 0, 0,
                               -1.0, 3, 1, 1, 0, None, 0, None, None, 0, None)
  assert rc == _lib.ERR_INVALID
  assert "'bandwidth' should have a positive value" in _lib.last_error()
