"""ksig_signature_kern_static: the entry point that allocates nothing.

It serves callers that cannot allocate device memory (an FFI host holding
only raw device pointers, a framework whose allocator owns the device
memory, a loop that cannot take cudaMalloc's device-wide synchronisation):
its scratch is a fixed 16 MiB array inside the library.  This file is named
to be collected last.  Its test calls the entry point through the C ABI
twice in a row, on different inputs, and checks each result against
ksig_signature_kern, which uses a caller workspace, at the DP tolerance of
the other parity tests (1e-5 relative).  The second call catches state left
behind by the first.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _walks(seed, n, L, d):
  rng = np.random.default_rng(seed)
  return np.cumsum(rng.standard_normal((n, L, d)) * 0.2, axis=1).astype(np.float32)


def _rel(a, b):
  a = a.double().cpu().numpy()
  b = b.double().cpu().numpy()
  return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def test_static_scratch_entry_matches_workspace_entry():
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as L
  lib = L.lib()
  fn = lib.ksig_signature_kern_static
  stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
  for call, (seed, nx, ny, Lx, Ly) in enumerate([(1, 9, 7, 60, 45), (2, 6, 11, 230, 90)]):
    X = torch.as_tensor(_walks(seed, nx, Lx, 3), device='cuda')
    Y = torch.as_tensor(_walks(seed + 10, ny, Ly, 3), device='cuda')
    Xs, Ys = E.Seqs(X), E.Seqs(Y)
    ref = E.sig_levels(Xs, Ys, L.PAIRS_FULL, 4, 1, True, L.STATIC_RBF, 0.8)
    out = torch.full_like(ref, float('nan'))
    rc = fn(ctypes.c_void_p(X.data_ptr()), None, nx, Lx,
            ctypes.c_void_p(Y.data_ptr()), None, ny, Ly, 3, L.DTYPE_F32,
            L.STATIC_RBF, 0.8, 4, 1, 1, L.PAIRS_FULL, None, 0,
            ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == L.OK, L.last_error()
    torch.cuda.synchronize()
    assert torch.isfinite(out).all(), f'call {call}: unwritten output'
    assert _rel(out, ref) < TOL, f'call {call}'


def test_static_scratch_entry_rejects_oversized_calls():
  from ksig_b200 import _lib as L
  lib = L.lib()
  X = torch.zeros((512, 1024, 16), device='cuda')
  out = torch.empty((3, 512 * 512), dtype=torch.float64, device='cuda')
  rc = lib.ksig_signature_kern_static(
      ctypes.c_void_p(X.data_ptr()), None, 512, 1024,
      ctypes.c_void_p(X.data_ptr()), None, 512, 1024, 16, L.DTYPE_F32,
      L.STATIC_RBF, 1.0, 2, 1, 1, L.PAIRS_FULL, None, 0,
      ctypes.c_void_p(out.data_ptr()), None)
  assert rc == L.ERR_WORKSPACE
  assert 'static scratch' in L.last_error()
