"""ctypes binding of ``lib/libksig_b200.so`` (declared in include/ksig_b200.h).

The library is the product: there is no CPU or PyTorch fallback.  Loading
fails loudly when the library has not been built (``python -m
ksig_b200.build``) or when no CUDA device is present at call time.
"""

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'lib', 'libksig_b200.so')

OK = 0
ERR_INVALID = 1
ERR_UNSUPPORTED = 2
ERR_WORKSPACE = 3
ERR_CUDA = 4
ERR_DEVICE = 5

STATIC_RBF = 0
STATIC_LINEAR = 1
STATIC_POLY = 2
STATIC_MATERN12 = 3
STATIC_MATERN32 = 4
STATIC_MATERN52 = 5
STATIC_RQ = 6
DTYPE_F32 = 0
DTYPE_F64 = 1
PAIRS_FULL = 0
PAIRS_UPPER = 1
PAIRS_DIAG = 2
PAIRS_LIST = 3

_lock = threading.Lock()
_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t

_SIGNATURES = {
    'ksig_version': (ctypes.c_char_p, []),
    'ksig_last_error': (_SZ, [ctypes.c_char_p, _SZ]),
    'ksig_num_pairs': (ctypes.c_longlong, [_I, _I, _I, _I]),
    'ksig_signature_kern_workspace': (_SZ, [_I] * 11),
    'ksig_signature_kern': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I, _I, _I,
                                 _D, _I, _I, _I, _I, _P, _I, _P, _P, _SZ,
                                 _P]),
    'ksig_signature_kern_pde_workspace': (_SZ, [_I] * 10),
    'ksig_signature_kern_pde': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I, _I,
                                     _I, _D, _I, _I, _I, _P, _I, _P, _P, _SZ,
                                     _P]),
    'ksig_normalize_levels': (_I, [_P, _I, _I, _I, _I, _P, _P, _I, _P, _I,
                                   _P]),
    'ksig_workspace_status': (_I, [_P, _P]),
    'ksig_static_status': (_I, [_P]),
    'ksig_signature_kern_bwd_workspace': (_SZ, [_I] * 11),
    'ksig_signature_kern_bwd': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I, _I,
                                     _I, _D, _I, _I, _I, _I, _P, _I, _P, _P,
                                     _P, _P, _SZ, _P]),
    'ksig_signature_kern_rec_workspace': (_SZ, [_I] * 11),
    'ksig_signature_kern_rec_fwd': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I,
                                         _I, _I, _D, _I, _I, _I, _I, _P, _I,
                                         _P, _P, _SZ, _P]),
    'ksig_signature_kern_rec_bwd': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I,
                                         _I, _I, _D, _I, _I, _I, _I, _P, _I,
                                         _P, _P, _P, _P, _SZ, _P]),
    'ksig_signature_kern_pde_bwd_workspace': (_SZ, [_I] * 10),
    'ksig_signature_kern_pde_bwd': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I,
                                         _I, _I, _D, _I, _I, _I, _P, _I, _P,
                                         _P, _P, _P, _SZ, _P]),
    'ksig_signature_kern_plain_workspace': (_SZ, [_I] * 10),
    'ksig_signature_kern_plain': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I, _I,
                                       _I, _D, _I, _I, _I, _P, _I, _P, _P, _SZ,
                                       _P]),
    'ksig_signature_kern_plain_bwd_workspace': (_SZ, [_I] * 10),
    'ksig_signature_kern_plain_bwd': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I,
                                           _I, _I, _D, _I, _I, _I, _P, _I, _P,
                                           _P, _P, _P, _SZ, _P]),
    'ksig_tune_set_cols': (_I, [_I, _I]),
    'ksig_tune_get_cols': (_I, [_I]),
    'ksig_signature_kern_ex': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I, _I,
                                    _I, _P, _I, _I, _I, _I, _P, _I, _P, _P,
                                    _SZ, _P]),
    'ksig_signature_kern_pde_ex': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I,
                                        _I, _I, _P, _I, _I, _I, _P, _I, _P,
                                        _P, _SZ, _P]),
    'ksig_global_align_kern_workspace': (_SZ, [_I] * 8),
    'ksig_global_align_kern': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I, _I,
                                    _I, _D, _I, _P, _I, _P, _P, _SZ, _P]),
    'ksig_launch_count': (ctypes.c_ulonglong, []),
    'ksig_profile_enable': (None, [_I]),
    'ksig_profile_read': (_I, [ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_longlong)]),
    'ksig_fp32_peak': (_I, [ctypes.POINTER(ctypes.c_double), _P]),
}

# Optional entry points bound when the library exports them.
_OPTIONAL = {
    'ksig_signature_kern_static': (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _I,
                                        _I, _I, _D, _I, _I, _I, _I, _P, _I,
                                        _P, _P]),
}


class KsigError(RuntimeError):
  """A failing ksig_b200 library call (code + message)."""

  def __init__(self, code, msg):
    super().__init__(f'ksig_b200 error {code}: {msg}')
    self.code = code


def lib():
  """Loads (once) and returns the ctypes library handle."""
  global _lib
  if _lib is not None:
    return _lib
  with _lock:
    if _lib is None:
      if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f'ksig_b200 CUDA library not found at {LIB_PATH}; build it with '
            '`python -m ksig_b200.build` (needs nvcc for sm_100a)')
      h = ctypes.CDLL(LIB_PATH)
      for name, (res, args) in _SIGNATURES.items():
        fn = getattr(h, name)
        fn.restype = res
        fn.argtypes = args
      for name, (res, args) in _OPTIONAL.items():
        fn = getattr(h, name, None)
        if fn is not None:
          fn.restype = res
          fn.argtypes = args
      _lib = h
  return _lib


def last_error():
  buf = ctypes.create_string_buffer(1024)
  lib().ksig_last_error(buf, 1024)
  return buf.value.decode(errors='replace')


def check(rc):
  """Raises for a non-zero status: ValueError for invalid arguments (the
  reference's exception type, ksig/utils.py:33-34), KsigError otherwise."""
  if rc == OK:
    return
  msg = last_error()
  if rc == ERR_INVALID:
    raise ValueError(msg)
  raise KsigError(rc, msg)


def exported_symbols():
  """Names of every entry point declared in include/ksig_b200.h."""
  return list(_SIGNATURES)
