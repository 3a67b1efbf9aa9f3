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


@pytest.mark.parametrize('dtype', ['f32', 'f64'])
def test_static_scratch_entry_ragged(dtype):
  """Ragged lengths (natural task order, lengths resolved in the shared
  array) and the FP64 path, two calls in a row, against
  ksig_signature_kern; then a length outside [1, L] is clamped, flagged in
  the array's status word and reported by ksig_static_status."""
  from ksig_b200 import _engine as E
  from ksig_b200 import _lib as L
  lib = L.lib()
  tdt = torch.float32 if dtype == 'f32' else torch.float64
  code = L.DTYPE_F32 if dtype == 'f32' else L.DTYPE_F64
  tol = TOL if dtype == 'f32' else 1e-10
  stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
  for call, (seed, nx, ny, Lx, Ly) in enumerate([(3, 5, 4, 70, 50), (4, 3, 6, 40, 300)]):
    X = torch.as_tensor(_walks(seed, nx, Lx, 2), device='cuda').to(tdt)
    Y = torch.as_tensor(_walks(seed + 5, ny, Ly, 2), device='cuda').to(tdt)
    rng = np.random.default_rng(seed)
    lx = torch.tensor(rng.integers(1, Lx + 1, nx), dtype=torch.int32, device='cuda')
    ly = torch.tensor(rng.integers(1, Ly + 1, ny), dtype=torch.int32, device='cuda')
    Xs, Ys = E.Seqs(X, lx), E.Seqs(Y, ly)
    ref = E.sig_levels(Xs, Ys, L.PAIRS_FULL, 3, 2, True, L.STATIC_RBF, 0.7)
    out = torch.full_like(ref, float('nan'))
    rc = lib.ksig_signature_kern_static(
        ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(lx.data_ptr()), nx, Lx,
        ctypes.c_void_p(Y.data_ptr()), ctypes.c_void_p(ly.data_ptr()), ny, Ly, 2, code,
        L.STATIC_RBF, 0.7, 3, 2, 1, L.PAIRS_FULL, None, 0,
        ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == L.OK, L.last_error()
    assert lib.ksig_static_status(stream) == L.OK
    assert torch.isfinite(out).all(), f'call {call}: unwritten output'
    assert _rel(out, ref) < tol, f'call {call}'
  # A length past L: clamped on the device and reported.
  bad = torch.tensor([Lx + 5] + [2] * (nx - 1), dtype=torch.int32, device='cuda')
  rc = lib.ksig_signature_kern_static(
      ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(bad.data_ptr()), nx, Lx,
      ctypes.c_void_p(Y.data_ptr()), None, ny, Ly, 2, code,
      L.STATIC_RBF, 0.7, 3, 2, 1, L.PAIRS_FULL, None, 0,
      ctypes.c_void_p(out.data_ptr()), stream)
  assert rc == L.OK
  assert lib.ksig_static_status(stream) == L.ERR_INVALID
  assert lib.ksig_static_status(stream) == L.OK  # read and cleared


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
