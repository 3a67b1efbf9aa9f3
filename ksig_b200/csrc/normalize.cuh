// Per-level normalisation and level mean of SignatureKernel._K
// (ksig/kernels.py:190-214): every level is divided by
// max(robust_sqrt(K_l(x,x)), eps) * max(robust_sqrt(K_l(y,y)), eps) with
// robust_sqrt(v) = sqrt(max(v, eps)) (ksig/utils.py:173-182), eps = 1e-12,
// and the levels are averaged.  Without normalisation the levels are summed
// (the reference's return_levels=False result).  All arithmetic in FP64.
#pragma once

#include "common.cuh"

namespace ksig {

struct NormArgs {
  const double* levels;  // [n_lev, P]
  int n_lev, mode, nX, nY;
  const double* dx;      // [n_lev, nX] or nullptr (diagonal of levels)
  const double* dy;      // [n_lev, nY] or nullptr
  int normalize;
};

__device__ __forceinline__ long long upper_index(long long a, long long b, long long n) {
  return a * n - a * (a - 1) / 2 + (b - a);
}

template <typename O>
__global__ void normalize_kernel(NormArgs a, O* __restrict__ out) {
  const long long total = (long long)a.nX * a.nY;
  const bool up = a.mode == KSIG_PAIRS_UPPER;
  const long long P = up ? (long long)a.nX * (a.nX + 1) / 2 : total;
  const double eps = 1e-12;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx / a.nY, j = idx - i * a.nY;
    const long long p = up ? (i <= j ? upper_index(i, j, a.nX) : upper_index(j, i, a.nX)) : idx;
    const long long pi = up ? upper_index(i, i, a.nX) : i * a.nY + i;
    const long long pj = up ? upper_index(j, j, a.nX) : j * a.nY + j;
    double acc = 0.0;
    for (int l = 0; l < a.n_lev; ++l) {
      const double v = a.levels[l * P + p];
      if (a.normalize) {
        const double kx = a.dx ? a.dx[(long long)l * a.nX + i] : a.levels[l * P + pi];
        const double ky = a.dy ? a.dy[(long long)l * a.nY + j] : a.levels[l * P + pj];
        const double sx = fmax(sqrt(fmax(kx, eps)), eps);
        const double sy = fmax(sqrt(fmax(ky, eps)), eps);
        acc += v / (sx * sy);
      } else {
        acc += v;
      }
    }
    out[idx] = (O)(a.normalize ? acc / a.n_lev : acc);
  }
}

}  // namespace ksig
