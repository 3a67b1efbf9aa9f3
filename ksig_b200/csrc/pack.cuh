// Packing of input sequences into the fused-Gram row format.
//
// A static-kernel value between point x (row side) and point y (column side)
// is evaluated by the hot kernels from packed rows of KD coordinates plus a
// norm slot at index KD:
//   RBF    (ksig/static/kernels.py:258-260, ksig/utils.py:149-156): both
//          sides raw (x, 0) and (y, 0).  The kernels move each lane's points
//          to a lane-centred frame (rbf_center_cols / rbf_center_row in
//          common.cuh) and evaluate arg = -a |x - y|^2 with
//          a = log2(e)/max(2s^2,1e-12), M = exp2(arg).
//   linear (ksig/static/kernels.py:155): xr = (s x, 0), yr = (y, 0),
//          arg = xr[KD] + yr[KD] + sum_{k<KD} xr[k] * yr[k], M = arg.
//   polynomial: as linear with s = 1 (arg = <x, y>); Matern / rational
//          quadratic: xr = (2x, -|x|^2), yr = (y, -|y|^2); their sweep
//          instantiations sum the squared distance from coordinate
//          differences, and static_value (common.cuh) forms the kernel value.
// Rows are padded with zeros to KD coordinates and to a 16-byte stride so the
// kernels read them with vector loads.  Norms are formed in FP64.
#pragma once

#include "common.cuh"

namespace ksig {

struct PackArgs {
  const void* src;      // [n, L, d] dense, dtype src_f64 ? double : float
  const int32_t* len;   // [n] or nullptr (= L)
  int n, L, d;
  int src_f64;
  int kind;             // KIND_RBF / KIND_LINEAR
  double param;         // bandwidth or scale
  int row_side;         // 1: x-side scaling, 0: y-side
  int kd;               // padded coordinate count (>= d)
  int stride;           // packed row stride in elements
  int32_t* len_out;     // [n] resolved lengths (clamped to [1, L])
  int* status;
};

template <typename T>
__global__ void pack_rows_kernel(PackArgs a, T* __restrict__ dst) {
  const long long total = (long long)a.n * a.L;
  const bool dist = kind_is_distance(a.kind);
  const bool raw = a.kind == KIND_RBF;  // centred in the kernels
  const double lin = a.kind == KIND_LINEAR ? a.param : 1.0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < total;
       r += (long long)gridDim.x * blockDim.x) {
    const int seq = (int)(r / a.L);
    const int t = (int)(r - (long long)seq * a.L);
    if (t == 0 && a.len_out) {
      int l = a.len ? a.len[seq] : a.L;
      if (l < 1 || l > a.L) set_status(a.status, KSIG_ERR_INVALID);
      a.len_out[seq] = l < 1 ? 1 : (l > a.L ? a.L : l);
    }
    T* out = dst + r * a.stride;
    double nrm = 0.0;
    for (int k = 0; k < a.kd; ++k) {
      double v = 0.0;
      if (k < a.d) {
        v = a.src_f64 ? ((const double*)a.src)[r * a.d + k]
                      : (double)((const float*)a.src)[r * a.d + k];
      }
      nrm += v * v;
      double o;
      if (raw) o = v;
      else if (dist) o = a.row_side ? 2.0 * v : v;
      else o = a.row_side ? lin * v : v;
      out[k] = (T)o;
    }
    out[a.kd] = (T)(dist && !raw ? -nrm : 0.0);
    for (int k = a.kd + 1; k < a.stride; ++k) out[k] = (T)0;
  }
}

}  // namespace ksig
