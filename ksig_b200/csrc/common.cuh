// Shared device helpers for the ksig_b200 signature-kernel library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ksig_b200.h"

namespace ksig {

constexpr unsigned FULL = 0xffffffffu;

// Static-kernel epilogue selector (ksig/static/kernels.py:245-260 RBF,
// :134-155 linear).
enum StaticKind : int {
  KIND_RBF = KSIG_STATIC_RBF,
  KIND_LINEAR = KSIG_STATIC_LINEAR,
  KIND_POLY = KSIG_STATIC_POLY,            // ksig/static/kernels.py:183-194
  KIND_MATERN12 = KSIG_STATIC_MATERN12,    // :263-277
  KIND_MATERN32 = KSIG_STATIC_MATERN32,    // :280-296
  KIND_MATERN52 = KSIG_STATIC_MATERN52,    // :299-316
  KIND_RQ = KSIG_STATIC_RQ,                // :319-343
};

// Kernels whose packed argument is minus the squared distance.
__host__ __device__ inline bool kind_is_distance(int kind) {
  return kind == KIND_RBF || kind == KIND_MATERN12 || kind == KIND_MATERN32 ||
         kind == KIND_MATERN52 || kind == KIND_RQ;
}

// Epilogue constants of a static kernel, formed on the host (capi.cu,
// static_params).
struct StaticParams {
  double c0, c1, c2;
};

// Device-side status word: kernels never trap; they record the first error
// code here and return.  The host reads it after the launch.
__device__ __forceinline__ void set_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

template <typename T> struct Vec;        // 16-byte vector of T
template <> struct Vec<float> { using type = float4; static constexpr int N = 4; };
template <> struct Vec<double> { using type = double2; static constexpr int N = 2; };

// exp2 in the compute type.  The float path maps to the hardware ex2 unit.
__device__ __forceinline__ float kexp2(float a) { return exp2f(a); }
__device__ __forceinline__ double kexp2(double a) { return exp2(a); }

// Fused-Gram argument of two packed rows, x[KD] + y[KD] + sum_{k<KD} x[k] y[k]
// (the packed format: norms at index KD, zero padding after it).  PAIR (FP32,
// KD >= 5) uses paired FP32 instructions (FFMA2: two fused multiply-adds per
// issue, each rounded like fmaf) over coordinate pairs (2j, 2j+1), summed in
// two interleaved chains that meet at the end.  It saves issue slots but
// can raise register use, so the kernels enable it per instantiation where
// their occupancy stays the same.
template <int KD, bool PAIR, typename XA, typename YA>
__device__ __forceinline__ float packed_arg(const XA& x, const YA& y, float) {
  if constexpr (PAIR && KD >= 5) {
    float2 s;
    if constexpr (KD % 2 == 1) {
      s = make_float2(x[KD] + y[KD], x[KD - 1] * y[KD - 1]);
#pragma unroll
      for (int j = 0; j < KD / 2; ++j)
        s = __ffma2_rn(make_float2(x[2 * j], x[2 * j + 1]), make_float2(y[2 * j], y[2 * j + 1]), s);
      return s.x + s.y;
    } else {
      s = __fmul2_rn(make_float2(x[0], x[1]), make_float2(y[0], y[1]));
#pragma unroll
      for (int j = 1; j < KD / 2; ++j)
        s = __ffma2_rn(make_float2(x[2 * j], x[2 * j + 1]), make_float2(y[2 * j], y[2 * j + 1]), s);
      return s.x + (s.y + (x[KD] + y[KD]));
    }
  } else {
    float acc = x[KD] + y[KD];
#pragma unroll
    for (int k = 0; k < KD; ++k) acc = fmaf(x[k], y[k], acc);
    return acc;
  }
}
template <int KD, bool PAIR, typename XA, typename YA>
__device__ __forceinline__ double packed_arg(const XA& x, const YA& y, double) {
  double acc = x[KD] + y[KD];
#pragma unroll
  for (int k = 0; k < KD; ++k) acc = fma(x[k], y[k], acc);
  return acc;
}

// Static kernel value from the fused dot-product argument (RBF, linear).
template <typename T>
__device__ __forceinline__ T static_value(T arg, int kind) {
  return kind == KIND_RBF ? kexp2(arg) : arg;
}

// Static kernel values of the other kinds, evaluated by their own sweep
// instantiations (EXT = true).  `arg` is <x, y> for the polynomial kernel
// and minus the squared distance D2 = |x-y|^2 for the others:
//   polynomial  c2 (arg + c0)^c1                  (scale, gamma, degree)
//   Matern12    exp(-D),  D = sqrt(max(D2, 1e-12)) c0,  c0 = 1 / max(s, eps)
//   Matern32    (1 + D) exp(-D),  same D with c0 = sqrt(3) / max(s, eps)
//   Matern52    (1 + D + E/3) exp(-D),  E = c0 D2, D = sqrt(max(E, 1e-12)),
//               c0 = 5 / max(s^2, eps)
//   RQ          (1 + c0 D2)^-c1,  c0 = 1 / max(2 a s^2, eps), c1 = a
// Matern12 / 32 use the distance between x and y; the reference's
// euclid_dist (ksig/utils.py:186-197) takes a stray `self` argument and
// measures within the second set instead, which this does not reproduce.
template <typename T>
__device__ __forceinline__ T static_value_other(T arg, int kind, const StaticParams& sp) {
  switch (kind) {
    case KIND_POLY: return T(sp.c2) * pow(arg + T(sp.c0), T(sp.c1));
    case KIND_MATERN12: {
      const T D = sqrt(fmax(-arg, T(1e-12))) * T(sp.c0);
      return exp(-D);
    }
    case KIND_MATERN32: {
      const T D = sqrt(fmax(-arg, T(1e-12))) * T(sp.c0);
      return (T(1) + D) * exp(-D);
    }
    case KIND_MATERN52: {
      const T E = -arg * T(sp.c0);
      const T D = sqrt(fmax(E, T(1e-12)));
      return (T(1) + D + E * (T(1) / T(3))) * exp(-D);
    }
    case KIND_RQ: return pow(T(1) + (-arg) * T(sp.c0), -T(sp.c1));
    default: return arg;
  }
}

template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) { return __shfl_up_sync(FULL, v, d); }
template <typename T>
__device__ __forceinline__ T shfl_down(T v, int d) { return __shfl_down_sync(FULL, v, d); }
template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int d) { return __shfl_xor_sync(FULL, v, d); }

__host__ __device__ constexpr int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Row stride (elements) of a packed point row holding KD coordinates plus the
// norm term, padded to a 16-byte multiple.
template <typename T>
__host__ __device__ constexpr int packed_stride(int kd) {
  return round_up(kd + 1, (int)(16 / sizeof(T)));
}

// Decodes a task index into a (row sequence, column sequence) pair.
// mode: KSIG_PAIRS_FULL (a*nY+b), KSIG_PAIRS_UPPER (a<=b, row-major upper
// triangle), KSIG_PAIRS_DIAG (a,a), KSIG_PAIRS_LIST (explicit int2 list).
__device__ __forceinline__ int2 decode_task(int t, int mode, int nY,
                                            const int2* list, const int* order) {
  if (order) t = order[t];
  if (mode == KSIG_PAIRS_LIST) return list[t];
  if (mode == KSIG_PAIRS_DIAG) return make_int2(t, t);
  if (mode == KSIG_PAIRS_FULL) return make_int2(t / nY, t % nY);
  // Upper triangle of an n x n grid, row-major: row a holds n - a entries.
  // Invert t = a*n - a*(a-1)/2 + (b - a) with a float estimate + fix-up.
  const int n = nY;
  double nn = 2.0 * n + 1.0;
  int a = (int)floor((nn - sqrt(nn * nn - 8.0 * (double)t)) * 0.5);
  if (a < 0) a = 0;
  if (a > n - 1) a = n - 1;
  auto start = [n](long long r) { return r * n - r * (r - 1) / 2; };
  while (a > 0 && start(a) > t) --a;
  while (a < n - 1 && start(a + 1) <= t) ++a;
  int b = a + (int)(t - start(a));
  return make_int2(a, b);
}

}  // namespace ksig
