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

// ---- RBF arguments in a lane-centred frame --------------------------------
// RBF rows are packed raw (x itself, norm slot zero).  A lane that owns the
// grid columns y_0 .. y_{C-1} of a strip (plus, in the adjoints, the next
// lane's first column y_C) moves the origin to its own first point c = y_0:
//   column slot 0:      -c                       (norm slot 0)
//   column slot c >= 1: (2a (y_c - c), -a |y_c - c|^2)
// and a grid row x becomes x' = x - c with norm slot -a |x'|^2, so that
//   arg_0 = -a |x'|^2,   arg_c = x'[KD] + y_c[KD] + sum_k x'_k y_c[k]
// (centred_arg on the transformed rows) is -a |x - y_c|^2 with a =
// log2(e) / max(2 s^2, 1e-12) (ksig/static/kernels.py:258-260).  The columns
// of one lane lie within a few steps of c, so |y_c - c| is small; then
// |x'|^2 + |y'|^2 - 2 <x', y'> cannot cancel (|x'| near |y'| means both are
// small), unlike |x|^2 + |y|^2 - 2 <x, y> for long unnormalised paths, where
// both norms reach 1e4 in FP32.  Column 0 needs no dot product at all.

// Pairwise sum of N values (a balanced tree: rounding error grows with
// log2 N, not N).
template <int N, typename T>
__device__ __forceinline__ T pair_sum(const T (&v)[N]) {
  T s[N];
#pragma unroll
  for (int i = 0; i < N; ++i) s[i] = v[i];
#pragma unroll
  for (int w = 1; w < N; w *= 2)
#pragma unroll
    for (int i = 0; i + w < N; i += 2 * w) s[i] += s[i + w];
  return s[0];
}

// Raw column points y[c][0..KD] (slot KD zero) -> lane-centred form; slot 0
// is the centre.  NC columns in a [NC][KD + 1] array.
template <int KD, int NC, typename T>
__device__ __forceinline__ void rbf_center_cols(T (&y)[NC][KD + 1], T alpha) {
  const T two_a = T(2) * alpha;
#pragma unroll
  for (int c = 1; c < NC; ++c) {
    T n = T(0);
#pragma unroll
    for (int k = 0; k < KD; ++k) {
      const T v = y[c][k] - y[0][k];
      n = fma(v, v, n);
      y[c][k] = two_a * v;
    }
    y[c][KD] = -alpha * n;
  }
#pragma unroll
  for (int k = 0; k < KD; ++k) y[0][k] = -y[0][k];
  y[0][KD] = T(0);
}

// One column of the lane-centred form from its raw point and the raw centre
// (for column storage outside a register array).
template <int KD, typename YA, typename CA, typename T>
__device__ __forceinline__ void rbf_center_col(YA& y, const CA& c0, T alpha) {
  const T two_a = T(2) * alpha;
  T n = T(0);
#pragma unroll
  for (int k = 0; k < KD; ++k) {
    const T v = y[k] - c0[k];
    n = fma(v, v, n);
    y[k] = two_a * v;
  }
  y[KD] = -alpha * n;
}

// Grid row x (raw) -> x' = x + negc (negc = column slot 0) with the norm
// slot -a |x'|^2; xt may alias x.  Scalar FADD / FFMA: the paired forms
// (FADD2 / FFMA2) were 5 % slower in the 512 x 512 sweep on B200, which
// spent the saved issue slots on register moves to form the pairs.
template <int KD, typename XA, typename NA>
__device__ __forceinline__ void rbf_center_row(const XA& x, const NA& negc, float alpha,
                                               float* xt) {
  float n = 0.f;
#pragma unroll
  for (int k = 0; k < KD; ++k) {
    const float v = x[k] + negc[k];
    xt[k] = v;
    n = fmaf(v, v, n);
  }
  xt[KD] = -alpha * n;
}
template <int KD, typename XA, typename NA>
__device__ __forceinline__ void rbf_center_row(const XA& x, const NA& negc, double alpha,
                                               double* xt) {
  double n = 0.0;
#pragma unroll
  for (int k = 0; k < KD; ++k) {
    const double v = x[k] + negc[k];
    xt[k] = v;
    n = fma(v, v, n);
  }
  xt[KD] = -alpha * n;
}

// RBF argument of a centred row x' (rbf_center_row) and a centred column y
// (rbf_center_cols): y[KD] + sum_k x'_k y_k + xnorm, with the row's norm
// term xnorm = x'[KD] added last, so that the dot-product chains do not
// wait for the norm chain of the same row.  PAIR as in packed_arg.
template <int KD, bool PAIR, typename XA, typename YA>
__device__ __forceinline__ float centred_arg(const XA& x, const YA& y, float xnorm) {
  if constexpr (PAIR && KD >= 5) {
    float2 s;
    if constexpr (KD % 2 == 1) {
      s = make_float2(y[KD], x[KD - 1] * y[KD - 1]);
#pragma unroll
      for (int j = 0; j < KD / 2; ++j)
        s = __ffma2_rn(make_float2(x[2 * j], x[2 * j + 1]), make_float2(y[2 * j], y[2 * j + 1]), s);
      return (s.x + s.y) + xnorm;
    } else {
      s = make_float2(y[KD], 0.f);
#pragma unroll
      for (int j = 0; j < KD / 2; ++j)
        s = __ffma2_rn(make_float2(x[2 * j], x[2 * j + 1]), make_float2(y[2 * j], y[2 * j + 1]), s);
      return (s.x + s.y) + xnorm;
    }
  } else {
    float acc = y[KD];
#pragma unroll
    for (int k = 0; k < KD; ++k) acc = fmaf(x[k], y[k], acc);
    return acc + xnorm;
  }
}
template <int KD, bool PAIR, typename XA, typename YA>
__device__ __forceinline__ double centred_arg(const XA& x, const YA& y, double xnorm) {
  double acc = y[KD];
#pragma unroll
  for (int k = 0; k < KD; ++k) acc = fma(x[k], y[k], acc);
  return acc + xnorm;
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
