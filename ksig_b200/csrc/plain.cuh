// Plain FP32 one-pair-per-block form of the truncated signature kernel: the
// comparison baseline for the fused sweep (no reference counterpart as a
// kernel; it is the reference's recursion, ksig/algorithms.py:47-140,
// written as a direct CUDA translation).
//
// One CTA per pair.  The CTA materialises the second-difference array Z
// (lx x ly, ksig/algorithms.py:63-64) in per-CTA global scratch from the
// packed points, then evaluates every level with the reference's array
// operations: exclusive cumulative sums along rows (one warp per row, warp
// scans) and along columns (one thread per column), the elementwise
// products, and a block reduction of the level total.  Everything is FP32
// except the final per-level reduction (FP64).  Order p (Alg. 6) keeps its
// p x p state arrays in scratch as the reference does.
#pragma once

#include "common.cuh"

namespace ksig {

template <typename T>
struct PlainArgs {
  const T* xr;           // packed row-side points  [*, RS]
  const int64_t* xstart;
  const int32_t* xlen;
  const T* yr;
  const int64_t* ystart;
  const int32_t* ylen;
  int rs, kd;            // packed row stride and coordinate count
  int mode, nY;
  const int2* list;
  int ntasks, nX, nYseq;
  int kind;
  int n_levels, order;   // order already clamped (1..n_levels)
  double* out;           // [n_levels+1, ntasks]
  T* scratch;            // per CTA: (2 + 2 p^2) arrays of cap floats
  long long cap;         // floats per array (>= max lx * ly)
  int* status;
};

template <typename T>
__device__ T block_sum(T v, T* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  T t = T(0);
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : T(0);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
  }
  return t;  // valid in thread 0
}

// dst(i,j) = sum_{j'<j} src(i,j') (exclusive along rows), one warp per row.
template <typename T>
__device__ void excl_rows(const T* src, T* dst, int lx, int ly) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwp = blockDim.x >> 5;
  for (int i = w; i < lx; i += nwp) {
    T carry = T(0);
    for (int j0 = 0; j0 < ly; j0 += 32) {
      const int j = j0 + lane;
      T v = j < ly ? src[(long long)i * ly + j] : T(0);
      T incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      if (j < ly) dst[(long long)i * ly + j] = carry + incl - v;
      carry += __shfl_sync(FULL, incl, 31);
    }
  }
}

// dst(i,j) = sum_{i'<i} src(i',j) (exclusive along columns), one thread per
// column; src == dst allowed.
template <typename T>
__device__ void excl_cols(const T* src, T* dst, int lx, int ly) {
  for (int j = threadIdx.x; j < ly; j += blockDim.x) {
    T acc = T(0);
    for (int i = 0; i < lx; ++i) {
      const T v = src[(long long)i * ly + j];
      dst[(long long)i * ly + j] = acc;
      acc += v;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) plain_dp_kernel(const PlainArgs<T> a) {
  __shared__ T sh[32];
  const long long per = a.cap;
  const int p = a.order;
  T* Z = a.scratch + (long long)blockIdx.x * per * (2 + 2 * p * p);
  T* tmp = Z + per;
  T* Rc = tmp + per;             // current level states  [p*p][cap]
  T* Rn = Rc + per * p * p;      // next level states
  for (int t = blockIdx.x; t < a.ntasks; t += gridDim.x) {
    const int2 ab = decode_task(t, a.mode, a.nY, a.list, nullptr);
    if (ab.x < 0 || ab.x >= a.nX || ab.y < 0 || ab.y >= a.nYseq) {
      if (threadIdx.x == 0) set_status(a.status, KSIG_ERR_INVALID);
      continue;
    }
    const int Lx = a.xlen[ab.x], Ly = a.ylen[ab.y];
    const int lx = Lx - 1, ly = Ly - 1;
    double* out = a.out;
    if (lx <= 0 || ly <= 0 || (long long)lx * ly > per) {
      if ((long long)lx * ly > per && threadIdx.x == 0) set_status(a.status, KSIG_ERR_DEVICE);
      if (threadIdx.x == 0)
        for (int k = 0; k <= a.n_levels; ++k) out[(long long)k * a.ntasks + t] = k == 0 ? 1.0 : 0.0;
      continue;
    }
    const T* xb = a.xr + a.xstart[ab.x] * a.rs;
    const T* yb = a.yr + a.ystart[ab.y] * a.rs;
    // Z(i,j) = M(i+1,j+1) - M(i+1,j) - M(i,j+1) + M(i,j), M from the points.
    auto Mv = [&](int i, int j) {
      const T* x = xb + (long long)i * a.rs;
      const T* y = yb + (long long)j * a.rs;
      T acc = x[a.kd] + y[a.kd];
      for (int k = 0; k < a.kd; ++k) acc = fma(x[k], y[k], acc);
      return static_value(acc, a.kind);
    };
    for (long long e = threadIdx.x; e < (long long)lx * ly; e += blockDim.x) {
      const int i = (int)(e / ly), j = (int)(e - (long long)i * ly);
      Z[e] = Mv(i + 1, j + 1) - Mv(i + 1, j) - Mv(i, j + 1) + Mv(i, j);
    }
    __syncthreads();
    const long long n = (long long)lx * ly;
    // Level 1.
    T part = T(0);
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
      part += Z[e];
      Rc[e] = Z[e];
    }
    T s = block_sum(part, sh);
    if (threadIdx.x == 0) { out[t] = 1.0; out[a.ntasks + t] = (double)s; }
    int dcur = 1;
    for (int k = 2; k <= a.n_levels; ++k) {
      const int d = k < p ? k : p;
      // R_next[0][0] = Z * excl2d(sum R).
      for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        T v = T(0);
        for (int q = 0; q < dcur * dcur; ++q) {
          const int r = q / dcur, c = q - r * dcur;
          v += Rc[(long long)(r * p + c) * per + e];
        }
        tmp[e] = v;
      }
      __syncthreads();
      excl_rows(tmp, tmp, lx, ly);
      __syncthreads();
      excl_cols(tmp, tmp, lx, ly);
      __syncthreads();
      for (long long e = threadIdx.x; e < n; e += blockDim.x) Rn[e] = Z[e] * tmp[e];
      __syncthreads();
      for (int r = 1; r < d; ++r) {
        // R_next[0][r] = Z/(r+1) * excl_cols(sum_a R[a][r-1]).
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = T(0);
          for (int q = 0; q < dcur; ++q) v += Rc[(long long)(q * p + (r - 1)) * per + e];
          tmp[e] = v;
        }
        __syncthreads();
        excl_cols(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          Rn[(long long)(0 * p + r) * per + e] = Z[e] * tmp[e] / T(r + 1);
        __syncthreads();
        // R_next[r][0] = Z/(r+1) * excl_rows(sum_b R[r-1][b]).
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = T(0);
          for (int q = 0; q < dcur; ++q) v += Rc[(long long)((r - 1) * p + q) * per + e];
          tmp[e] = v;
        }
        __syncthreads();
        excl_rows(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          Rn[(long long)(r * p + 0) * per + e] = Z[e] * tmp[e] / T(r + 1);
        for (int c = 1; c < d; ++c)
          for (long long e = threadIdx.x; e < n; e += blockDim.x)
            Rn[(long long)(r * p + c) * per + e] =
                Z[e] * Rc[(long long)((r - 1) * p + (c - 1)) * per + e] / T((r + 1) * (c + 1));
        __syncthreads();
      }
      // Level total, then the next level's states become current.
      part = T(0);
      for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        T v = T(0);
        for (int q = 0; q < d * d; ++q) {
          const int r = q / d, c = q - r * d;
          const T rv = Rn[(long long)(r * p + c) * per + e];
          v += rv;
          Rc[(long long)(r * p + c) * per + e] = rv;
        }
        part += v;
      }
      s = block_sum(part, sh);
      if (threadIdx.x == 0) out[(long long)k * a.ntasks + t] = (double)s;
      __syncthreads();
      dcur = d;
    }
    __syncthreads();
  }
}

}  // namespace ksig
