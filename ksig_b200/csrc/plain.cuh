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
  T ralpha;              // RBF: log2(e) / max(2 s^2, 1e-12)
};

// Static-kernel argument of two packed points (pack.cuh): RBF rows are raw,
// arg = -a |x - y|^2; linear arg = <s x, y>.
template <typename T>
__device__ __forceinline__ T plain_arg(const T* x, const T* y, int kd, int kind, T ralpha) {
  T acc = T(0);
  if (kind == KIND_RBF) {
    for (int k = 0; k < kd; ++k) {
      const T v = x[k] - y[k];
      acc = fma(v, v, acc);
    }
    return -ralpha * acc;
  }
  for (int k = 0; k < kd; ++k) acc = fma(x[k], y[k], acc);
  return acc;
}

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
      return static_value(plain_arg(x, y, a.kd, a.kind, a.ralpha), a.kind);
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

// ---------------------------------------------------------------------------
// Plain FP32 one-pair-per-block adjoint: the baseline of the fused skewed
// backward sweep.  One CTA per pair keeps Z, every level's states and the
// adjoint states as full lx x ly arrays in per-CTA scratch and evaluates the
// adjoint of ksig/algorithms.py:88-140 with array passes:
//   Rbar_{k-1}[a][b] = w_{k-1} + S2^T(Z Rbar_k[0][0])
//                      + Sc^T(Z/(b+2) Rbar_k[0][b+1]) + Sr^T(Z/(a+2) Rbar_k[a+1][0])
//                      + Z/((a+2)(b+2)) Rbar_k[a+1][b+1],
//   Zbar += sum_{r,s} Rbar_k[r][s] dR_k[r][s]/dZ,
// (S^T: exclusive suffix sums over both axes, columns (i) or rows (j)),
// then Mbar = the transposed second difference of Zbar and dX, dparam by
// per-row reductions over the grid.
// ---------------------------------------------------------------------------

template <typename T>
struct PlainBwdArgs {
  PlainArgs<T> f;        // inputs, enumeration, scratch (per CTA: nbuf * cap)
  const double* glev;    // [nl_out + 1, ntasks]
  int nl_out;
  T* dX;                 // [nX, LX, d]
  int LX, d;
  double param;
  double* dparam;        // may be null
  int nbuf;              // arrays per CTA
};

// dst(i,j) = sum_{j'>j} src(i,j') (exclusive suffix along rows), one warp
// per row; src == dst allowed.
template <typename T>
__device__ void suf_rows(const T* src, T* dst, int lx, int ly) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwp = blockDim.x >> 5;
  for (int i = w; i < lx; i += nwp) {
    T carry = T(0);
    for (int j1 = ly; j1 > 0; j1 -= 32) {
      const int j = j1 - 1 - lane;
      T v = j >= 0 ? src[(long long)i * ly + j] : T(0);
      T incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      if (j >= 0) dst[(long long)i * ly + j] = carry + incl - v;
      carry += __shfl_sync(FULL, incl, 31);
    }
  }
}

// dst(i,j) = sum_{i'>i} src(i',j) (exclusive suffix along columns).
template <typename T>
__device__ void suf_cols(const T* src, T* dst, int lx, int ly) {
  for (int j = threadIdx.x; j < ly; j += blockDim.x) {
    T acc = T(0);
    for (int i = lx - 1; i >= 0; --i) {
      const T v = src[(long long)i * ly + j];
      dst[(long long)i * ly + j] = acc;
      acc += v;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) plain_dp_bwd_kernel(const PlainBwdArgs<T> ba) {
  const PlainArgs<T>& a = ba.f;
  const long long per = a.cap;
  const int p = a.order, NL = a.n_levels;
  auto fdim = [&](int k) { return k < p ? k : p; };
  // Level-k state (r, s) lives at array base(k) + r * f(k) + s.
  auto base = [&](int k) {
    int b = 0;
    for (int q = 1; q < k; ++q) b += fdim(q) * fdim(q);
    return b;
  };
  T* buf = a.scratch + (long long)blockIdx.x * per * ba.nbuf;
  T* Z = buf;
  T* R = Z + per;                                   // all level states
  T* Rb = R + per * base(NL + 1);                   // adjoint of level k   [p*p]
  T* Rn = Rb + per * p * p;                         // adjoint of level k-1 [p*p]
  T* Zb = Rn + per * p * p;
  T* tmp = Zb + per;
  T* Wg = tmp + per;                                // grid weights, Lx * Ly
  const double alpha = 1.4426950408889634 / fmax(2.0 * ba.param * ba.param, 1e-12);
  const bool rbf = a.kind == KIND_RBF;
  for (int t = blockIdx.x; t < a.ntasks; t += gridDim.x) {
    const int2 ab = decode_task(t, a.mode, a.nY, a.list, nullptr);
    if (ab.x < 0 || ab.x >= a.nX || ab.y < 0 || ab.y >= a.nYseq) {
      if (threadIdx.x == 0) set_status(a.status, KSIG_ERR_INVALID);
      continue;
    }
    const int Lx = a.xlen[ab.x], Ly = a.ylen[ab.y];
    const int lx = Lx - 1, ly = Ly - 1;
    if (lx <= 0 || ly <= 0) continue;
    if ((long long)Lx * Ly > per) {
      if (threadIdx.x == 0) set_status(a.status, KSIG_ERR_DEVICE);
      continue;
    }
    const long long n = (long long)lx * ly;
    const T* xb = a.xr + a.xstart[ab.x] * a.rs;
    const T* yb = a.yr + a.ystart[ab.y] * a.rs;
    auto argv = [&](int i, int j) {
      const T* x = xb + (long long)i * a.rs;
      const T* y = yb + (long long)j * a.rs;
      return plain_arg(x, y, a.kd, a.kind, a.ralpha);
    };
    auto Mv = [&](int i, int j) { return static_value(argv(i, j), a.kind); };
    auto wk = [&](int k) {
      return (k >= 1 && k <= ba.nl_out) ? (T)ba.glev[(long long)k * a.ntasks + t] : T(0);
    };
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
      const int i = (int)(e / ly), j = (int)(e - (long long)i * ly);
      Z[e] = Mv(i + 1, j + 1) - Mv(i + 1, j) - Mv(i, j + 1) + Mv(i, j);
    }
    __syncthreads();
    // ---- forward: all level states ----
    for (long long e = threadIdx.x; e < n; e += blockDim.x) R[e] = Z[e];
    __syncthreads();
    for (int k = 2; k <= NL; ++k) {
      const int d = fdim(k), dp = fdim(k - 1);
      const T* Rc = R + per * base(k - 1);
      T* Rk = R + per * base(k);
      for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        T v = T(0);
        for (int q = 0; q < dp * dp; ++q) v += Rc[(long long)q * per + e];
        tmp[e] = v;
      }
      __syncthreads();
      excl_rows(tmp, tmp, lx, ly);
      __syncthreads();
      excl_cols(tmp, tmp, lx, ly);
      __syncthreads();
      for (long long e = threadIdx.x; e < n; e += blockDim.x) Rk[e] = Z[e] * tmp[e];
      __syncthreads();
      for (int r = 1; r < d; ++r) {
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = T(0);
          for (int q = 0; q < dp; ++q) v += Rc[(long long)(q * dp + (r - 1)) * per + e];
          tmp[e] = v;
        }
        __syncthreads();
        excl_cols(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          Rk[(long long)(0 * d + r) * per + e] = Z[e] * tmp[e] / T(r + 1);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = T(0);
          for (int q = 0; q < dp; ++q) v += Rc[(long long)((r - 1) * dp + q) * per + e];
          tmp[e] = v;
        }
        __syncthreads();
        excl_rows(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          Rk[(long long)(r * d + 0) * per + e] = Z[e] * tmp[e] / T(r + 1);
        for (int c = 1; c < d; ++c)
          for (long long e = threadIdx.x; e < n; e += blockDim.x)
            Rk[(long long)(r * d + c) * per + e] =
                Z[e] * Rc[(long long)((r - 1) * dp + (c - 1)) * per + e] / T((r + 1) * (c + 1));
        __syncthreads();
      }
    }
    // ---- adjoint, top level down ----
    {
      const int d = fdim(NL);
      const T w = wk(NL);
      for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        Zb[e] = T(0);
        for (int q = 0; q < d * d; ++q) Rb[(long long)q * per + e] = w;
      }
      __syncthreads();
    }
    for (int k = NL; k >= 1; --k) {
      const int d = fdim(k);
      if (k == 1) {
        for (long long e = threadIdx.x; e < n; e += blockDim.x) Zb[e] += Rb[e];
        __syncthreads();
        break;
      }
      const int dp = fdim(k - 1);
      const T* Rc = R + per * base(k - 1);
      // Zbar += Rbar_k[0][0] * excl2d(sum R_{k-1}).
      for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        T v = T(0);
        for (int q = 0; q < dp * dp; ++q) v += Rc[(long long)q * per + e];
        tmp[e] = v;
      }
      __syncthreads();
      excl_rows(tmp, tmp, lx, ly);
      __syncthreads();
      excl_cols(tmp, tmp, lx, ly);
      __syncthreads();
      for (long long e = threadIdx.x; e < n; e += blockDim.x) Zb[e] += Rb[e] * tmp[e];
      __syncthreads();
      for (int r = 1; r < d; ++r) {
        // [0][r]: excl_cols(sum_a R_{k-1}[a][r-1]) / (r+1)
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = T(0);
          for (int q = 0; q < dp; ++q) v += Rc[(long long)(q * dp + (r - 1)) * per + e];
          tmp[e] = v;
        }
        __syncthreads();
        excl_cols(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          Zb[e] += Rb[(long long)(0 * p + r) * per + e] * tmp[e] / T(r + 1);
        __syncthreads();
        // [r][0]: excl_rows(sum_b R_{k-1}[r-1][b]) / (r+1)
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = T(0);
          for (int q = 0; q < dp; ++q) v += Rc[(long long)((r - 1) * dp + q) * per + e];
          tmp[e] = v;
        }
        __syncthreads();
        excl_rows(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          T v = Rb[(long long)(r * p + 0) * per + e] * tmp[e] / T(r + 1);
          for (int c = 1; c < d; ++c)
            v += Rb[(long long)(r * p + c) * per + e] *
                 Rc[(long long)((r - 1) * dp + (c - 1)) * per + e] / T((r + 1) * (c + 1));
          Zb[e] += v;
        }
        __syncthreads();
      }
      // Rbar_{k-1}: every state gets w_{k-1} + S2^T(Z Rbar_k[0][0]).
      for (long long e = threadIdx.x; e < n; e += blockDim.x) tmp[e] = Z[e] * Rb[e];
      __syncthreads();
      suf_rows(tmp, tmp, lx, ly);
      __syncthreads();
      suf_cols(tmp, tmp, lx, ly);
      __syncthreads();
      {
        const T w = wk(k - 1);
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          for (int q = 0; q < dp * dp; ++q) Rn[(long long)q * per + e] = w + tmp[e];
      }
      __syncthreads();
      for (int r = 1; r < d; ++r) {
        // R_k[0][r] reads column prefixes of R_{k-1}[a][r-1].
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          tmp[e] = Z[e] * Rb[(long long)(0 * p + r) * per + e] / T(r + 1);
        __syncthreads();
        suf_cols(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          for (int q = 0; q < dp; ++q) Rn[(long long)(q * dp + (r - 1)) * per + e] += tmp[e];
        __syncthreads();
        // R_k[r][0] reads row prefixes of R_{k-1}[r-1][b].
        for (long long e = threadIdx.x; e < n; e += blockDim.x)
          tmp[e] = Z[e] * Rb[(long long)(r * p + 0) * per + e] / T(r + 1);
        __syncthreads();
        suf_rows(tmp, tmp, lx, ly);
        __syncthreads();
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
          for (int q = 0; q < dp; ++q) Rn[(long long)((r - 1) * dp + q) * per + e] += tmp[e];
          for (int c = 1; c < d; ++c)
            Rn[(long long)((r - 1) * dp + (c - 1)) * per + e] +=
                Z[e] * Rb[(long long)(r * p + c) * per + e] / T((r + 1) * (c + 1));
        }
        __syncthreads();
      }
      // The level k-1 adjoint becomes current (re-indexed to stride p).
      for (long long e = threadIdx.x; e < n; e += blockDim.x)
        for (int r = 0; r < dp; ++r)
          for (int c = 0; c < dp; ++c)
            Rb[(long long)(r * p + c) * per + e] = Rn[(long long)(r * dp + c) * per + e];
      __syncthreads();
    }
    // ---- Mbar on the grid and the pull-back into dX, dparam ----
    const int Gx = Lx, Gy = Ly;
    auto zb = [&](int i, int j) -> T {
      return (i >= 0 && i < lx && j >= 0 && j < ly) ? Zb[(long long)i * ly + j] : T(0);
    };
    double dpl = 0.0;
    for (long long e = threadIdx.x; e < (long long)Gx * Gy; e += blockDim.x) {
      const int i = (int)(e / Gy), j = (int)(e - (long long)i * Gy);
      const T mb = zb(i - 1, j - 1) - zb(i - 1, j) - zb(i, j - 1) + zb(i, j);
      const T ar = argv(i, j);
      const T Wv = rbf ? mb * kexp2(ar) : mb;
      Wg[e] = Wv;
      if (ba.dparam) dpl += rbf ? (double)Wv * (-(double)ar / alpha) : (double)Wv * (double)ar;
    }
    __syncthreads();
    const double sc = rbf ? 1.0 / (ba.param * ba.param) : ba.param;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nwp = blockDim.x >> 5;
    for (int i = wp; i < Gx; i += nwp) {
      const T* xr = xb + (long long)i * a.rs;
      for (int k = 0; k < ba.d; ++k) {
        T acc = T(0), sw = T(0);
        for (int j = lane; j < Gy; j += 32) {
          const T Wv = Wg[(long long)i * Gy + j];
          acc = fma(Wv, yb[(long long)j * a.rs + k], acc);
          sw += Wv;
        }
        for (int o = 16; o > 0; o >>= 1) {
          acc += __shfl_xor_sync(FULL, acc, o);
          sw += __shfl_xor_sync(FULL, sw, o);
        }
        if (lane == 0) {
          const T v = rbf ? acc - sw * xr[k] : acc;
          atomicAdd(ba.dX + ((long long)ab.x * ba.LX + i) * ba.d + k, (T)(sc * (double)v));
        }
      }
    }
    if (ba.dparam) {
      for (int o = 16; o > 0; o >>= 1) dpl += __shfl_xor_sync(FULL, dpl, o);
      __shared__ double shd[32];
      __syncthreads();
      if (lane == 0) shd[wp] = dpl;
      __syncthreads();
      if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < nwp; ++q) s += shd[q];
        const double pp = ba.param;
        atomicAdd(ba.dparam, rbf ? s / (pp * pp * pp) : s / pp);
      }
    }
    __syncthreads();
  }
}

}  // namespace ksig
