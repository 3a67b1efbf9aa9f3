// Shared device helpers for the ksig_b200 signature-kernel library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ksig_b200.h"

namespace ksig {

constexpr unsigned FULL = 0xffffffffu;

// Static-kernel epilogue selector (ksig/static/kernels.py:245-260 RBF,
// :134-155 linear).
enum StaticKind : int { KIND_RBF = KSIG_STATIC_RBF, KIND_LINEAR = KSIG_STATIC_LINEAR };

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

// Static kernel value from the fused dot-product argument.
template <typename T>
__device__ __forceinline__ T static_value(T arg, int kind) {
  return kind == KIND_RBF ? kexp2(arg) : arg;
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
