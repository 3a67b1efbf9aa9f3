// Adjoint of the Goursat-PDE signature kernel (no reference counterpart: the
// reference has no gradients).
//
// Forward scheme per refined cell (ksig/algorithms.py:384-385, q = Z / F^2):
//   K[i+1,j+1] = A (K[i,j+1] + K[i+1,j]) - B K[i,j],
//   A = 1 + q/2 + q^2/12, B = 1 - q^2/12, output K[N, M].
// Exact discrete adjoint: with L = w K[N, M], Lam = dL/dK satisfies
//   Lam[i,j] = A(i,j-1) Lam[i+1,j] + A(i-1,j) Lam[i,j+1] - B(i,j) Lam[i+1,j+1]
// (coefficients of the refined cell named; cells outside the grid give 0),
// Lam[N,M] = w, and
//   dL/dq(i,j) = Lam[i+1,j+1] ((K[i,j+1] + K[i+1,j]) (1/2 + q/6) + K[i,j] q/6).
// On the grid reversed in both axes, G(a,b) = Lam[N-a, M-b] obeys a
// forward-type scheme
//   G(a,b) = Ar G(a-1,b) + Ab G(a,b-1) - B G(a-1,b-1)
// whose B comes from the point's own (reversed) cell and whose Ar / Ab come
// from the cells above and to the left of it, with zero boundaries and the
// seed G(0,0) = w.  Both passes therefore run as the forward kernel does:
// lanes own column blocks, lane l one row step behind lane l-1, and the
// update in increment form (H = vertical increment accumulated along the
// row) that keeps FP32 rounding small.
//
// Phase 1 (per pair): reversed sweep; G is stored to per-warp scratch.
// Phase 2: forward sweep over the original grid; each refined cell reads
// Lam[i+1,j+1] = G(N-1-i, M-1-j) and adds dL/dZ of its cell.  Zbar is
// pulled back through the second difference -- each lane takes the part of
// Mbar that comes from its own cells, and the parts of neighbouring lanes
// add up to the full Mbar -- and through the static kernel into dX (one
// grid row per lane per step, atomics) and dparam.
#pragma once

#include "common.cuh"

namespace ksig {

template <typename T>
struct PdeBwdArgs {
  const T* xr;
  const int64_t* xstart;
  const int32_t* xlen;
  const T* yr;
  const int64_t* ystart;
  const int32_t* ylen;
  int mode, nY;
  const int2* list;
  const int* order;       // optional task permutation (longest first)
  int ntasks, nX, nYseq;
  int kind;
  double param;
  const double* grad;     // [ntasks] dL/dK per pair
  T* dX;                  // [nX, LX, d] row-side gradient (accumulated)
  int LX, d;
  double* dparam;         // may be null
  T* scratch;             // per warp: G grid, then the strip boundary buffer
  long long scratch_per_warp;
  long long grid_stride;  // row stride of G (>= refined columns)
  long long bb_off;       // offset of the boundary buffer in a warp's scratch
  int rows_max;           // cell rows the boundary buffer holds
  int* status;
};

// W-wide vector of T (W * sizeof(T) <= 16) for the adjoint-grid traffic.
template <typename T, int W> struct VecW;
template <> struct VecW<float, 1> { using type = float; };
template <> struct VecW<float, 2> { using type = float2; };
template <> struct VecW<float, 4> { using type = float4; };
template <> struct VecW<double, 1> { using type = double; };
template <> struct VecW<double, 2> { using type = double2; };

template <typename T, int KD, int C, int F, int WPB>
__global__ void __launch_bounds__(WPB * 32)
pde_bwd_kernel(const PdeBwdArgs<T> args) {
  // A lane's F refined columns of one cell are contiguous in G (reversed in
  // phase 2), so they move as W-wide vectors: the grid row base and the
  // per-warp scratch are 16-byte aligned and F * (cell column) is a
  // multiple of W.
  constexpr int GW0 = 16 / (int)sizeof(T);
  constexpr int GW = F < GW0 ? F : GW0;
  using GV = typename VecW<T, GW>::type;
  constexpr int RS = packed_stride<T>(KD);
  constexpr int VN = Vec<T>::N;
  using V = typename Vec<T>::type;
  constexpr int STRIP = 32 * C - 1;
  constexpr int NXE = 2 * F + 2;  // per cell row: K, H per refined row, Z, Z(row above)
  constexpr T invF2 = T(1) / T(F * F);

  const int lane = threadIdx.x & 31;
  const long long wg = (long long)blockIdx.x * WPB + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * WPB;
  T* Gs = args.scratch + wg * args.scratch_per_warp;
  T* BB = Gs + args.bb_off;
  const long long GS = args.grid_stride;
  const double alpha = 1.4426950408889634 / fmax(2.0 * args.param * args.param, 1e-12);
  const bool rbf = args.kind == KIND_RBF;

  for (long long tid = wg; tid < args.ntasks; tid += nw) {
    const int2 ab = decode_task((int)tid, args.mode, args.nY, args.list, args.order);
    const int task = args.order ? args.order[tid] : (int)tid;
    if (ab.x < 0 || ab.x >= args.nX || ab.y < 0 || ab.y >= args.nYseq) {
      if (lane == 0) set_status(args.status, KSIG_ERR_INVALID);
      continue;
    }
    const int a = ab.x, b = ab.y;
    const int Lx = args.xlen[a], Ly = args.ylen[b];
    const int lx = Lx - 1, ly = Ly - 1;
    if (lx <= 0 || ly <= 0) continue;  // K = 1: no gradient
    const int ns = (ly + STRIP - 1) / STRIP;
    if (ns > 1 && lx > args.rows_max) {
      if (lane == 0) set_status(args.status, KSIG_ERR_DEVICE);
      continue;
    }
    const int N = lx * F, M = ly * F;
    const T w = (T)args.grad[task];
    const T* xb = args.xr + args.xstart[a] * RS;
    const T* yb = args.yr + args.ystart[b] * RS;

    // The lane's C+1 grid columns of strip s (phase 1: reversed grid).
    T yv[C + 1][KD + 1];
    auto load_y = [&](int s, bool rev) {
#pragma unroll
      for (int c = 0; c <= C; ++c) {
        int col = s * STRIP + C * lane + c;
        col = col < Ly - 1 ? col : Ly - 1;
        if (rev) col = Ly - 1 - col;
        const V* p = reinterpret_cast<const V*>(yb + (long long)col * RS);
        T tmp[RS];
#pragma unroll
        for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(tmp)[v] = __ldg(p + v);
#pragma unroll
        for (int k = 0; k <= KD; ++k) yv[c][k] = tmp[k];
      }
    };
    auto gram = [&](int row, bool rev, T (&m)[C + 1], T (&arg)[C + 1], T (&xv)[RS]) {
      row = row < Lx - 1 ? row : Lx - 1;
      if (rev) row = Lx - 1 - row;
      const V* p = reinterpret_cast<const V*>(xb + (long long)row * RS);
#pragma unroll
      for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(p + v);
#pragma unroll
      for (int c = 0; c <= C; ++c) {
        T acc = xv[KD] + yv[c][KD];
#pragma unroll
        for (int k = 0; k < KD; ++k) acc = fma(xv[k], yv[c][k], acc);
        arg[c] = acc;
        m[c] = static_value(acc, args.kind);
      }
    };

    // ------------------------- phase 1: reversed adjoint sweep -------------
    for (int s = 0; s < ns; ++s) {
      load_y(s, true);
      const int g0 = s * STRIP + C * lane;
      T Mlo[C + 1], Mhi[C + 1], argd[C + 1], xv[RS];
      gram(0, true, Mlo, argd, xv);
      T Kr[C * F];
#pragma unroll
      for (int j = 0; j < C * F; ++j) Kr[j] = T(0);
      T kcorner = T(0);
      T X[NXE];
#pragma unroll
      for (int h = 0; h < NXE; ++h) X[h] = T(0);
      T Zprev[C];
#pragma unroll
      for (int c = 0; c < C; ++c) Zprev[c] = T(0);
      for (int t = 0; t < lx + 32; ++t) {
        const int r = t - lane;  // reversed cell row of this lane
        T Xin[NXE];
#pragma unroll
        for (int h = 0; h < NXE; ++h) Xin[h] = shfl_up(X[h], 1);
        if (r >= 0 && r < lx) {
          gram(r + 1, true, Mhi, argd, xv);
          T Z[C];
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const bool valid = g0 + c < ly && !(lane == 31 && c == C - 1);
            Z[c] = valid ? (Mhi[c + 1] - Mhi[c] - Mlo[c + 1] + Mlo[c]) : T(0);
          }
          if (lane == 0) {
            if (s > 0) {
              const T* src = BB + (long long)r * NXE;
#pragma unroll
              for (int h = 0; h < NXE; ++h) Xin[h] = __ldcg(src + h);
            } else {
#pragma unroll
              for (int h = 0; h < NXE; ++h) Xin[h] = T(0);
              if (r == 0) Xin[F] = w;  // seed G(0,0) = w through the left H
            }
          }
          // Z of the cell columns left-extended by the left neighbour's cell.
          T Zx[C + 1], Zpx[C + 1];
          Zx[0] = Xin[2 * F];
          Zpx[0] = Xin[2 * F + 1];
#pragma unroll
          for (int c = 0; c < C; ++c) { Zx[c + 1] = Z[c]; Zpx[c + 1] = Zprev[c]; }
#pragma unroll
          for (int f = 0; f < F; ++f) {
            T klo = (f == 0) ? kcorner : Xin[f > 0 ? f - 1 : 0];
            T kln = Xin[f];
            T H = Xin[F + f];
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const bool skip = (c == C - 1) && lane == 31;
#pragma unroll
              for (int g = 0; g < F; ++g) {
                // Refined point (rF+f, (g0+c)F+g); its own cell is the refined
                // cell up-left of it, Ar the cell above, Ab the cell to the left.
                const T z_up = (f > 0) ? Zx[c + 1] : Zpx[c + 1];
                const T z_left = (g > 0) ? Zx[c + 1] : Zx[c];
                const T z_ul = (f > 0) ? z_left : ((g > 0) ? Zpx[c + 1] : Zpx[c]);
                const T qr = z_up * invF2, qb = z_left * invF2, qo = z_ul * invF2;
                const T ar = qr * fma(qr, T(1) / T(12), T(0.5));
                const T ab_ = qb * fma(qb, T(1) / T(12), T(0.5));
                const T bq = qo * qo * (T(1) / T(12));
                const int J = c * F + g;
                const T kro = Kr[J];
                const T gg = fma(ar, kro, fma(ab_, kln, bq * klo));
                const T Hn = H + gg;
                const T krn = kro + Hn;
                if (!skip) {
                  klo = kro;
                  kln = krn;
                  H = Hn;
                  Kr[J] = krn;
                }
              }
            }
            X[f] = kln;
            X[F + f] = H;
            // Store G at refined row rF+f for the lane's refined columns.
            const long long grow = (long long)r * F + f;
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const bool valid = g0 + c < ly && !(lane == 31 && c == C - 1);
              if (valid) {
                GV* dst = reinterpret_cast<GV*>(Gs + grow * GS + (long long)(g0 + c) * F);
#pragma unroll
                for (int v = 0; v < F / GW; ++v) {
                  GV gv;
                  T* e = reinterpret_cast<T*>(&gv);
#pragma unroll
                  for (int i = 0; i < GW; ++i) e[i] = Kr[c * F + v * GW + i];
                  __stcg(dst + v, gv);
                }
              }
            }
          }
          kcorner = Xin[F - 1];
          // Z of this lane's last valid cell (this row, row above) for the
          // lane to the right.
          X[2 * F] = (lane == 31) ? Z[C >= 2 ? C - 2 : 0] : Z[C - 1];
          X[2 * F + 1] = (lane == 31) ? Zprev[C >= 2 ? C - 2 : 0] : Zprev[C - 1];
          if (lane == 31 && s + 1 < ns) {
            T* dst = BB + (long long)r * NXE;
#pragma unroll
            for (int h = 0; h < NXE; ++h) __stcg(dst + h, X[h]);
          }
#pragma unroll
          for (int c = 0; c < C; ++c) Zprev[c] = Z[c];
#pragma unroll
          for (int c = 0; c <= C; ++c) Mlo[c] = Mhi[c];
        }
        __syncwarp();
      }
    }
    __syncwarp();

    // ------------------------- phase 2: forward + gradient ----------------
    double dpar = 0.0;
    const double scale_x = rbf ? 1.0 / (args.param * args.param) : args.param;
    for (int s = 0; s < ns; ++s) {
      load_y(s, false);
      const int g0 = s * STRIP + C * lane;
      T Mlo[C + 1], arglo[C + 1], Mhi[C + 1], arghi[C + 1], xlo[RS], xhi[RS];
      gram(0, false, Mlo, arglo, xlo);
      T Kr[C * F];
#pragma unroll
      for (int j = 0; j < C * F; ++j) Kr[j] = T(1);
      T kcorner = T(1);
      T X[NXE];
#pragma unroll
      for (int h = 0; h < NXE; ++h) X[h] = T(0);
      T Zbp[C];  // Zbar of the row above (this lane's cells)
#pragma unroll
      for (int c = 0; c < C; ++c) Zbp[c] = T(0);
      for (int t = 0; t < lx + 1 + 32; ++t) {
        const int r = t - lane;  // cell row of this lane; r == lx finishes grid row lx
        T Xin[NXE];
#pragma unroll
        for (int h = 0; h < NXE; ++h) Xin[h] = shfl_up(X[h], 1);
        if (r >= 0 && r <= lx) {
          T Zb[C];
#pragma unroll
          for (int c = 0; c < C; ++c) Zb[c] = T(0);
          if (r < lx) {
            gram(r + 1, false, Mhi, arghi, xhi);
            T Z[C];
#pragma unroll
            for (int c = 0; c < C; ++c) Z[c] = Mhi[c + 1] - Mhi[c] - Mlo[c + 1] + Mlo[c];
            if (lane == 0) {
              if (s > 0) {
                const T* src = BB + (long long)r * NXE;
#pragma unroll
                for (int h = 0; h < 2 * F; ++h) Xin[h] = __ldcg(src + h);
              } else {
#pragma unroll
                for (int f = 0; f < F; ++f) { Xin[f] = T(1); Xin[F + f] = T(0); }
              }
            }
            T a_[C], b_[C], qv[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const T q = Z[c] * invF2;
              qv[c] = q;
              b_[c] = q * q * (T(1) / T(12));
              a_[c] = fma(T(0.5), q, b_[c]);
            }
#pragma unroll
            for (int f = 0; f < F; ++f) {
              T klo = (f == 0) ? kcorner : Xin[f > 0 ? f - 1 : 0];
              T kln = Xin[f];
              T H = Xin[F + f];
              // Lam[i+1, j+1] = G(N-1-i, M-1-j) for refined row i = rF+f.
              const long long grow = (long long)(N - 1 - (r * F + f));
#pragma unroll
              for (int c = 0; c < C; ++c) {
                const bool skip = (c == C - 1) && lane == 31;
                const bool valid = g0 + c < ly && !skip;
                // Lam of the cell's F refined columns: G columns
                // M - (g0+c+1)F .. M - (g0+c)F - 1, in reverse.
                T lamv[F];
                if (valid) {
                  const GV* src = reinterpret_cast<const GV*>(
                      Gs + grow * GS + (long long)(M - (g0 + c + 1) * F));
#pragma unroll
                  for (int v = 0; v < F / GW; ++v) {
                    const GV gv = __ldcg(src + v);
                    const T* e = reinterpret_cast<const T*>(&gv);
#pragma unroll
                    for (int i = 0; i < GW; ++i) lamv[F - 1 - (v * GW + i)] = e[i];
                  }
                } else {
#pragma unroll
                  for (int g = 0; g < F; ++g) lamv[g] = T(0);
                }
#pragma unroll
                for (int g = 0; g < F; ++g) {
                  const int J = c * F + g;
                  const T kro = Kr[J];
                  const T gg = fma(kro + kln, a_[c], klo * b_[c]);
                  const T Hn = H + gg;
                  const T krn = kro + Hn;
                  if (valid) {
                    const T lam = lamv[g];
                    const T q6 = qv[c] * (T(1) / T(6));
                    Zb[c] = fma(lam, fma(kro + kln, T(0.5) + q6, klo * q6), Zb[c]);
                  }
                  if (!skip) {
                    klo = kro;
                    kln = krn;
                    H = Hn;
                    Kr[J] = krn;
                  }
                }
              }
              X[f] = kln;
              X[F + f] = H;
            }
            kcorner = Xin[F - 1];
            if (lane == 31 && s + 1 < ns) {
              T* dst = BB + (long long)r * NXE;
#pragma unroll
              for (int h = 0; h < 2 * F; ++h) __stcg(dst + h, X[h]);
            }
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const bool valid = g0 + c < ly && !((c == C - 1) && lane == 31);
              Zb[c] = valid ? Zb[c] * invF2 : T(0);
            }
          }
          // Grid row r: Mbar from this lane's cells of rows r-1 (Zbp) and r
          // (Zb), on the lane's grid columns g0 .. g0+C.
          T q[KD];
#pragma unroll
          for (int k = 0; k < KD; ++k) q[k] = T(0);
          T sw = T(0);
          const T inv2a = T(1) / T(2.0 * alpha);
#pragma unroll
          for (int c = 0; c <= C; ++c) {
            const T lo_l = (c > 0) ? Zb[c > 0 ? c - 1 : 0] : T(0);
            const T lo_r = (c < C) ? Zb[c < C ? c : 0] : T(0);
            const T hi_l = (c > 0) ? Zbp[c > 0 ? c - 1 : 0] : T(0);
            const T hi_r = (c < C) ? Zbp[c < C ? c : 0] : T(0);
            // Mbar(r, j) = Zbar(r-1, j-1) - Zbar(r-1, j) - Zbar(r, j-1) + Zbar(r, j)
            const T mbar = hi_l - hi_r - lo_l + lo_r;
            const bool col_ok = g0 + c < Ly;
            const T W = col_ok ? (rbf ? mbar * Mlo[c] : mbar) : T(0);
            sw += W;
#pragma unroll
            for (int k = 0; k < KD; ++k) q[k] = fma(W, yv[c][k], q[k]);
            if (col_ok)
              dpar += rbf ? (double)W * (-(double)arglo[c] / alpha) : (double)W * (double)Mlo[c];
          }
          if (rbf) {
#pragma unroll
            for (int k = 0; k < KD; ++k) q[k] -= sw * (xlo[k] * inv2a);
          }
          T* dst = args.dX + ((long long)a * args.LX + r) * args.d;
#pragma unroll
          for (int k = 0; k < KD; ++k)
            if (k < args.d && q[k] != T(0)) atomicAdd(dst + k, (T)(scale_x * (double)q[k]));
#pragma unroll
          for (int c = 0; c < C; ++c) Zbp[c] = Zb[c];
          if (r < lx) {
#pragma unroll
            for (int c = 0; c <= C; ++c) { Mlo[c] = Mhi[c]; arglo[c] = arghi[c]; }
#pragma unroll
            for (int k = 0; k < RS; ++k) xlo[k] = xhi[k];
          }
        }
        __syncwarp();
      }
    }
    if (args.dparam) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dpar += __shfl_xor_sync(FULL, dpar, o);
      if (lane == 0) {
        const double p = args.param;
        atomicAdd(args.dparam, rbf ? dpar / (p * p * p) : dpar / p);
      }
    }
  }
}

}  // namespace ksig
