// Static-kernel Gram of whole pairs, for the Gram-input sweep instantiations
// (KD == 0 in sweep.cuh) that serve any number of channels.
//
// The fused sweeps keep each lane's column points in registers, which caps
// the channel count they are compiled for.  Beyond it a call runs in chunks
// of tasks: this kernel writes the static-kernel values M(x_i, y_j) of every
// pair of a chunk into a [rows][ld] slot per task (ksig/static/kernels.py:
// 145-155, 183-194, 248-343 through ksig/utils.py:105-157), and the sweep
// then reads them in place of its register Gram.  The squared distance of
// the distance kernels is summed from coordinate differences (no
// |x|^2 + |y|^2 - 2 <x, y> cancellation), the polynomial and linear kernels
// from products.
//
// One CTA computes a 64 x 64 tile of one pair: 256 threads, 4 x 4 entries
// each (rows ty + 16 r, columns tx + 16 c, so each store instruction covers
// 16 consecutive columns), coordinates staged through shared memory 32 at a
// time.
#pragma once

#include "common.cuh"

namespace ksig {

template <typename T>
struct GramArgs {
  const T* xr;            // packed rows (pack.cuh), stride rs, kd coordinates
  const int64_t* xstart;
  const int32_t* xlen;
  const T* yr;
  const int64_t* ystart;
  const int32_t* ylen;
  int rs, kd;
  int mode, nY;           // pair enumeration (decode_task)
  const int2* list;
  const int* order;
  int task_base, ntasks;  // the slots of this launch: positions task_base ..
  int nX, nYseq;
  int kind;
  T ralpha;               // RBF: log2(e) / max(2 s^2, 1e-12)
  StaticParams sp;
  T* gram;                // [ntasks][rows][ld]
  long long slot;         // elements per slot
  int ld;                 // row stride of a slot
  int tiles_y;            // 64-column tiles per slot row
  int* status;
};

constexpr int kGramTile = 64;
constexpr int kGramKC = 32;

// MODE 0: raw rows, arg = -a |x - y|^2 (RBF); 1: rows packed as 2x,
// arg = -|x - y|^2 (Matern, rational quadratic); 2: arg = <x_r, y_r>
// (linear with the scale on the row side, polynomial).
template <typename T, int MODE>
__device__ __forceinline__ void gram_tile(const GramArgs<T>& a, int Lx, int Ly, int i0, int j0,
                                          const T* xb, const T* yb, T* out,
                                          T (&xs)[kGramTile][kGramKC + 1],
                                          T (&ys)[kGramTile][kGramKC + 1]) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = T(0);
  for (int k0 = 0; k0 < a.kd; k0 += kGramKC) {
    __syncthreads();
    for (int e = threadIdx.x; e < kGramTile * kGramKC; e += blockDim.x) {
      const int rr = e / kGramKC, kk = e - rr * kGramKC;
      const int k = k0 + kk;
      const int i = min(i0 + rr, Lx - 1), j = min(j0 + rr, Ly - 1);
      xs[rr][kk] = k < a.kd ? xb[(long long)i * a.rs + k] : T(0);
      ys[rr][kk] = k < a.kd ? yb[(long long)j * a.rs + k] : T(0);
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kGramKC; ++kk) {
      T xv[4], yv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) xv[r] = xs[ty + 16 * r][kk];
#pragma unroll
      for (int c = 0; c < 4; ++c) yv[c] = ys[tx + 16 * c][kk];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (MODE == 2) {
            acc[r][c] = fma(xv[r], yv[c], acc[r][c]);
          } else {
            const T v = MODE == 0 ? xv[r] - yv[c] : fma(T(0.5), xv[r], -yv[c]);
            acc[r][c] = fma(v, v, acc[r][c]);
          }
        }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i >= Lx) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = j0 + tx + 16 * c;
      if (j >= Ly) continue;
      T m;
      if (MODE == 0) m = kexp2(-a.ralpha * acc[r][c]);
      else if (MODE == 1) m = static_value_other(-acc[r][c], a.kind, a.sp);
      else m = a.kind == KIND_LINEAR ? acc[r][c] : static_value_other(acc[r][c], a.kind, a.sp);
      out[(long long)i * a.ld + j] = m;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) gram_kernel(const GramArgs<T> a) {
  const int slot = blockIdx.y;
  const int pos = a.task_base + slot;
  const int2 ab = decode_task(pos, a.mode, a.nY, a.list, a.order);
  if (ab.x < 0 || ab.x >= a.nX || ab.y < 0 || ab.y >= a.nYseq) {
    if (threadIdx.x == 0 && blockIdx.x == 0) set_status(a.status, KSIG_ERR_INVALID);
    return;
  }
  const int Lx = a.xlen[ab.x], Ly = a.ylen[ab.y];
  const int ti = blockIdx.x / a.tiles_y, tj = blockIdx.x - ti * a.tiles_y;
  const int i0 = ti * kGramTile, j0 = tj * kGramTile;
  if (i0 >= Lx || j0 >= Ly) return;  // the tile lies past this pair's lengths
  const T* xb = a.xr + a.xstart[ab.x] * a.rs;
  const T* yb = a.yr + a.ystart[ab.y] * a.rs;
  T* out = a.gram + (long long)slot * a.slot;
  __shared__ T xs[kGramTile][kGramKC + 1];
  __shared__ T ys[kGramTile][kGramKC + 1];
  if (a.kind == KIND_RBF) gram_tile<T, 0>(a, Lx, Ly, i0, j0, xb, yb, out, xs, ys);
  else if (kind_is_distance(a.kind)) gram_tile<T, 1>(a, Lx, Ly, i0, j0, xb, yb, out, xs, ys);
  else gram_tile<T, 2>(a, Lx, Ly, i0, j0, xb, yb, out, xs, ys);
}

}  // namespace ksig
