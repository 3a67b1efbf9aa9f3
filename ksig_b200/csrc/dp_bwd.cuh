// Adjoint of the truncated signature kernel (no reference counterpart: the
// reference has no gradients).  Gradients of the level kernels with respect
// to the row-side sequence of each pair and to the static-kernel parameter.
//
// Forward recursion (order 1 shown; order p analogous, ksig/algorithms.py:
// 47-140): R_1 = Z, R_k = Z * S(R_{k-1}), level_k = sum R_k with S the
// exclusive 2-D prefix (i' < i, j' < j).  For L = sum_k w_k level_k the
// adjoint is
//   Rbar_k = w_k + S^T(Z * Rbar_{k+1})     (S^T: suffix over i' > i, j' > j)
//   Zbar   = sum_k Rbar_k * S(R_{k-1})     (S(R_0) = 1)
// and for order p the row / column prefixes have suffix adjoints the same
// way.  Zbar is pulled back through the second difference
// (ksig/algorithms.py:63-64) to Mbar on the grid and through the static
// kernel (RBF: dM/dx = M (y - x) / s^2, dM/ds = M |x - y|^2 / s^3; linear:
// dM/dx = s y, dM/ds = M / s) into dX and dparam.
//
// One warp per pair, all lanes on the same cell row.  Phase 1 sweeps the
// rows top-down and keeps the final column sums (per strip).  Phase 2 sweeps
// bottom-up: it recovers every forward prefix at row i by subtracting row i
// from the column sums (no stored activations), forms the adjoint with
// column suffix sums held per lane and horizontal suffix sums from warp
// scans, and accumulates the gradient of grid row i+1.  Strips wider than
// 32*C-1 cells exchange per-row carries through global scratch.
#pragma once

#include "common.cuh"
#include "sweep.cuh"

namespace ksig {

template <typename T>
struct DpBwdArgs {
  const T* xr;           // packed row-side points  [*, RS]
  const int64_t* xstart;
  const int32_t* xlen;
  const T* yr;           // packed column-side points
  const int64_t* ystart;
  const int32_t* ylen;
  int mode, nY;
  const int2* list;
  int ntasks, nX, nYseq;
  int kind;
  double param;
  const double* glev;    // [nl_out + 1, ntasks] dL/dlevel (row 0 unused)
  int nl_out;
  T* dX;                 // [nX, LX, d] row-side gradient (accumulated)
  int LX, d;
  double* dparam;        // scalar (accumulated), may be null
  T* scratch;
  long long scratch_per_warp;
  int ns_max, rows_max;
  int* status;
};

// Inclusive warp scan (prefix over lanes 0..lane) of one value.
template <typename T>
__device__ __forceinline__ T warp_prefix_incl(T v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(FULL, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// Inclusive warp suffix scan (over lanes lane..31) of one value.
template <typename T>
__device__ __forceinline__ T warp_suffix_incl(T v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_down_sync(FULL, v, o);
    if (lane + o < 32) v += y;
  }
  return v;
}

// Reduces VP values (VP a power of two <= 32) over the warp; afterwards lane
// l holds the total of value index red_index<VP>(l).
template <int VP>
__device__ __forceinline__ int red_index(int lane) {
  int idx = 0, n = VP;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    if (n > 1) {
      n >>= 1;
      if (lane & o) idx += n;
    }
  }
  return idx;
}

template <typename T, int VP>
__device__ __forceinline__ T transpose_reduce(T (&v)[VP], int lane) {
  int n = VP;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    if (n > 1) {
      const int half = n >> 1;
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int i = 0; i < VP / 2; ++i) {
        if (i < half) {
          const T send = up ? v[i] : v[i + half];
          const T keep = up ? v[i + half] : v[i];
          v[i] = keep + __shfl_xor_sync(FULL, send, o);
        }
      }
      n = half;
    } else {
      v[0] += __shfl_xor_sync(FULL, v[0], o);
    }
  }
  return v[0];
}

template <int N>
struct Pow2Up { static constexpr int v = N <= 1 ? 1 : 2 * Pow2Up<(N + 1) / 2>::v; };
template <> struct Pow2Up<1> { static constexpr int v = 1; };

template <typename T, int KD, int C, int NL, int P, int WPB>
__global__ void __launch_bounds__(WPB * 32)
dp_bwd_kernel(const DpBwdArgs<T> args) {
  using Lay = DpLayout<NL, P>;
  constexpr int NX = Lay::NH > 0 ? Lay::NH : 1;
  constexpr int RS = packed_stride<T>(KD);
  constexpr int VN = Vec<T>::N;
  using V = typename Vec<T>::type;
  constexpr int STRIP = 32 * C - 1;
  constexpr int VP = Pow2Up<KD>::v;
  // Per-cell forward coefficients kept between the two passes of a row:
  // for level k the coefficient of Z in each state R_k[r][s].
  constexpr int NCOEF = 1 + (NL >= 2 ? (NL - 1) * P * P : 0);

  const int lane = threadIdx.x & 31;
  const long long wg = (long long)blockIdx.x * WPB + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * WPB;
  T* scr = args.scratch ? args.scratch + wg * args.scratch_per_warp : nullptr;
  // Scratch layout (multi-strip only): BL[ns_max][rows_max][NX] forward
  // carries, BR[rows_max][NX] adjoint carries, CS[ns_max][32][NX][C] final
  // column sums per strip.
  T* BL = scr;
  T* BR = scr ? scr + (long long)args.ns_max * args.rows_max * NX : nullptr;
  T* CS = scr ? BR + (long long)args.rows_max * NX : nullptr;

  const double alpha = 1.4426950408889634 / fmax(2.0 * args.param * args.param, 1e-12);
  const bool rbf = args.kind == KIND_RBF;

  for (long long tid = wg; tid < args.ntasks; tid += nw) {
    int2 ab = decode_task((int)tid, args.mode, args.nY, args.list, nullptr);
    if (ab.x < 0 || ab.x >= args.nX || ab.y < 0 || ab.y >= args.nYseq) {
      if (lane == 0) set_status(args.status, KSIG_ERR_INVALID);
      continue;
    }
    const int a = ab.x, b = ab.y;
    const int Lx = args.xlen[a], Ly = args.ylen[b];
    const int lx = Lx - 1, ly = Ly - 1;
    if (lx <= 0 || ly <= 0) continue;  // no cells: levels >= 1 are constant
    const int ns = (ly + STRIP - 1) / STRIP;
    if (ns > 1 && (!scr || ns > args.ns_max || lx > args.rows_max)) {
      if (lane == 0) set_status(args.status, KSIG_ERR_DEVICE);
      continue;
    }
    T w[NL + 1];
#pragma unroll
    for (int k = 0; k <= NL; ++k)
      w[k] = (k >= 1 && k <= args.nl_out) ? (T)args.glev[(long long)k * args.ntasks + tid] : T(0);

    const T* xb = args.xr + args.xstart[a] * RS;
    const T* yb = args.yr + args.ystart[b] * RS;
    T yv[C][KD + 1];
    auto load_y = [&](int s) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        int col = s * STRIP + C * lane + c;
        col = col < Ly - 1 ? col : Ly - 1;
        const V* p = reinterpret_cast<const V*>(yb + (long long)col * RS);
        T tmp[RS];
#pragma unroll
        for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(tmp)[v] = __ldg(p + v);
#pragma unroll
        for (int k = 0; k <= KD; ++k) yv[c][k] = tmp[k];
      }
    };
    auto load_x = [&](int row, T (&xv)[RS]) {
      row = row < Lx - 1 ? row : Lx - 1;
      const V* p = reinterpret_cast<const V*>(xb + (long long)row * RS);
#pragma unroll
      for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(p + v);
    };
    auto gram = [&](const T (&xv)[RS], T (&m)[C], T (&arg)[C]) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        T acc = xv[KD] + yv[c][KD];
#pragma unroll
        for (int k = 0; k < KD; ++k) acc = fma(xv[k], yv[c][k], acc);
        arg[c] = acc;
        m[c] = static_value(acc, args.kind);
      }
    };
    // Z of cell row r from grid rows r (Mlo) and r+1 (Mhi); masks the cell
    // that belongs to the next strip.
    auto cells = [&](const T (&Mlo)[C], const T (&Mhi)[C], T (&Z)[C]) {
      T DM[C];
#pragma unroll
      for (int c = 0; c < C; ++c) DM[c] = Mhi[c] - Mlo[c];
      const T right = shfl_down(DM[0], 1);
#pragma unroll
      for (int c = 0; c < C - 1; ++c) Z[c] = DM[c + 1] - DM[c];
      Z[C - 1] = lane == 31 ? T(0) : right - DM[C - 1];
    };

    T CC[NX][C];  // forward column sums (rows < i) of A / V inputs

    // ---------------- phase 1: forward, top-down, strips left to right -----
    for (int s = 0; s < ns; ++s) {
      load_y(s);
#pragma unroll
      for (int h = 0; h < NX; ++h)
#pragma unroll
        for (int c = 0; c < C; ++c) CC[h][c] = T(0);
      T xv[RS], Mlo[C], Mhi[C], argd[C];
      load_x(0, xv);
      gram(xv, Mlo, argd);
      for (int r = 0; r < lx; ++r) {
        load_x(r + 1, xv);
        gram(xv, Mhi, argd);
        T Z[C];
        cells(Mlo, Mhi, Z);
        // Carry-in of horizontal sums from the strip to the left.
        T carry[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h)
          carry[h] = (s > 0) ? BL[((long long)s * args.rows_max + r) * NX + h] : T(0);
        // 2-D prefixes: exclusive prefix over columns of CC (rows < r).
        T Hs[NX];  // per-lane exclusive carry for each horizontal quantity
        T tot[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h) {
          T t = T(0);
#pragma unroll
          for (int c = 0; c < C; ++c) t += CC[h][c];
          tot[h] = t;
        }
        // S2 parts (index off(k)) are known at row start; row-prefix parts
        // (off(k)+r') need this row's values and are scanned per level.
#pragma unroll
        for (int k = 2; k <= NL; ++k) {
          const int o = Lay::off(k);
          const T inc = warp_prefix_incl(tot[o], lane);
          Hs[o] = inc - tot[o] + carry[o];
          if (lane == 31 && s + 1 < ns) BL[((long long)(s + 1) * args.rows_max + r) * NX + o] = inc + carry[o];
        }
        // Per-cell recursion with per-level row-prefix scans.
        T Rst[C][P][P];
        T Utot[P];
#pragma unroll
        for (int c = 0; c < C; ++c) {
#pragma unroll
          for (int i = 0; i < P; ++i)
#pragma unroll
            for (int j = 0; j < P; ++j) Rst[c][i][j] = T(0);
          Rst[c][0][0] = Z[c];
        }
#pragma unroll
        for (int k = 2; k <= NL; ++k) {
          const int f = Lay::f(k), fp = Lay::f(k - 1), o = Lay::off(k);
          // Row prefixes of U_r (current row values of the previous level).
          T Uv[C][P];
#pragma unroll
          for (int rr = 1; rr < P; ++rr) {
            if (rr < f) {
              T t = T(0);
#pragma unroll
              for (int c = 0; c < C; ++c) {
                T u = T(0);
#pragma unroll
                for (int i = 0; i < P; ++i)
                  if (i < fp) u += Rst[c][rr - 1][i];
                Uv[c][rr] = u;
                t += u;
              }
              Utot[rr] = t;
              const T inc = warp_prefix_incl(t, lane);
              Hs[o + rr] = inc - t + carry[o + rr];
              if (lane == 31 && s + 1 < ns)
                BL[((long long)(s + 1) * args.rows_max + r) * NX + o + rr] = inc + carry[o + rr];
            }
          }
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const T z = Z[c];
            T A = T(0);
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
              for (int j = 0; j < P; ++j)
                if (i < fp && j < fp) A += Rst[c][i][j];
            T Rn[P][P];
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
              for (int j = 0; j < P; ++j) Rn[i][j] = T(0);
            Rn[0][0] = z * Hs[o];
            Hs[o] += CC[o][c];
            CC[o][c] += A;
#pragma unroll
            for (int rr = 1; rr < P; ++rr) {
              if (rr < f) {
                T Vs = T(0);
#pragma unroll
                for (int i = 0; i < P; ++i)
                  if (i < fp) Vs += Rst[c][i][rr - 1];
                const T zr = z * (T(1) / T(rr + 1));
                Rn[0][rr] = zr * CC[o + rr][c];
                CC[o + rr][c] += Vs;
                Rn[rr][0] = zr * Hs[o + rr];
                Hs[o + rr] += Uv[c][rr];
#pragma unroll
                for (int ss = 1; ss < P; ++ss)
                  if (ss < f)
                    Rn[rr][ss] = z * (T(1) / T((rr + 1) * (ss + 1))) * Rst[c][rr - 1][ss - 1];
              }
            }
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
              for (int j = 0; j < P; ++j) Rst[c][i][j] = Rn[i][j];
          }
        }
#pragma unroll
        for (int c = 0; c < C; ++c) Mlo[c] = Mhi[c];
      }
      if (ns > 1) {
        T* dst = CS + (((long long)s * 32 + lane) * NX) * C;
#pragma unroll
        for (int h = 0; h < NX; ++h)
#pragma unroll
          for (int c = 0; c < C; ++c) dst[h * C + c] = CC[h][c];
        __syncwarp();  // carries of lane 31 -> all lanes of the next strip
      }
    }

    // ---------------- phase 2: adjoint, bottom-up, strips right to left ----
    double dpar = 0.0;
    for (int s = ns - 1; s >= 0; --s) {
      load_y(s);
      if (ns > 1) {
        const T* src = CS + (((long long)s * 32 + lane) * NX) * C;
#pragma unroll
        for (int h = 0; h < NX; ++h)
#pragma unroll
          for (int c = 0; c < C; ++c) CC[h][c] = src[h * C + c];
      }
      T DA[NX][C];   // adjoint column suffix sums (rows > i)
#pragma unroll
      for (int h = 0; h < NX; ++h)
#pragma unroll
        for (int c = 0; c < C; ++c) DA[h][c] = T(0);
      const int g0 = s * STRIP + C * lane;
      T xv[RS], Mhi[C], arghi[C], Zbhi[C];
      load_x(lx, xv);
      gram(xv, Mhi, arghi);
#pragma unroll
      for (int c = 0; c < C; ++c) Zbhi[c] = T(0);
      T xhi[RS];
#pragma unroll
      for (int k = 0; k < RS; ++k) xhi[k] = xv[k];
      for (int r = lx - 1; r >= -1; --r) {
        T Mlo[C], arglo[C], Zb[C];
        T xlo[RS];
        if (r >= 0) {
          load_x(r, xlo);
          gram(xlo, Mlo, arglo);
          T Z[C];
          cells(Mlo, Mhi, Z);
          T carry[NX], bcarry[NX];
#pragma unroll
          for (int h = 0; h < NX; ++h) {
            carry[h] = (s > 0) ? BL[((long long)s * args.rows_max + r) * NX + h] : T(0);
            bcarry[h] = (s + 1 < ns) ? BR[(long long)r * NX + h] : T(0);
          }
          // ---- ascending: recover the forward prefixes at row r ----
          T coef[C][NCOEF];
          T Rst[C][P][P];
#pragma unroll
          for (int c = 0; c < C; ++c) {
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
              for (int j = 0; j < P; ++j) Rst[c][i][j] = T(0);
            Rst[c][0][0] = Z[c];
            coef[c][0] = T(1);
          }
#pragma unroll
          for (int k = 2; k <= NL; ++k) {
            const int f = Lay::f(k), fp = Lay::f(k - 1), o = Lay::off(k);
            const int cb = 1 + (k - 2) * P * P;
            // Column sums back to rows < r.
#pragma unroll
            for (int c = 0; c < C; ++c) {
              T A = T(0);
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j)
                  if (i < fp && j < fp) A += Rst[c][i][j];
              CC[o][c] -= A;
#pragma unroll
              for (int rr = 1; rr < P; ++rr) {
                if (rr < f) {
                  T Vs = T(0);
#pragma unroll
                  for (int i = 0; i < P; ++i)
                    if (i < fp) Vs += Rst[c][i][rr - 1];
                  CC[o + rr][c] -= Vs;
                }
              }
            }
            T t = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c) t += CC[o][c];
            T H2 = warp_prefix_incl(t, lane) - t + carry[o];
            T HU[P], Uv[C][P];
#pragma unroll
            for (int rr = 1; rr < P; ++rr) {
              HU[rr] = T(0);
              if (rr < f) {
                T tu = T(0);
#pragma unroll
                for (int c = 0; c < C; ++c) {
                  T u = T(0);
#pragma unroll
                  for (int i = 0; i < P; ++i)
                    if (i < fp) u += Rst[c][rr - 1][i];
                  Uv[c][rr] = u;
                  tu += u;
                }
                HU[rr] = warp_prefix_incl(tu, lane) - tu + carry[o + rr];
              }
            }
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const T z = Z[c];
              T cf[P][P];
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) cf[i][j] = T(0);
              cf[0][0] = H2;
              H2 += CC[o][c];
#pragma unroll
              for (int rr = 1; rr < P; ++rr) {
                if (rr < f) {
                  cf[0][rr] = CC[o + rr][c] * (T(1) / T(rr + 1));
                  cf[rr][0] = HU[rr] * (T(1) / T(rr + 1));
                  HU[rr] += Uv[c][rr];
#pragma unroll
                  for (int ss = 1; ss < P; ++ss)
                    if (ss < f) cf[rr][ss] = Rst[c][rr - 1][ss - 1] * (T(1) / T((rr + 1) * (ss + 1)));
                }
              }
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) {
                  coef[c][cb + i * P + j] = cf[i][j];
                  Rst[c][i][j] = z * cf[i][j];
                }
            }
          }
          // ---- descending: adjoint at row r ----
          // Horizontal suffixes of the column suffix sums DA (rows > r) for
          // the 2-D prefix adjoints, all levels at once.
          T Abar[NX];
#pragma unroll
          for (int k = 2; k <= NL; ++k) {
            const int o = Lay::off(k);
            T t = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c) t += DA[o][c];
            const T inc = warp_suffix_incl(t, lane);
            Abar[o] = inc - t + bcarry[o];
            if (lane == 0 && s > 0) BR[(long long)r * NX + o] = inc + bcarry[o];
          }
          T Rb_next[C][P][P];
          T Ub[P];
          // Column-suffix increments of the level processed last: they are
          // added to DA only after the next lower level has read DA, so that
          // every suffix used in row r covers rows > r only.
          T pendDA[P][C];
#pragma unroll
          for (int c = 0; c < C; ++c) Zb[c] = T(0);
#pragma unroll
          for (int k = NL; k >= 1; --k) {
            const int f = Lay::f(k);
            const int fn = (k < NL) ? Lay::f(k + 1) : 0;
            const int on = (k < NL) ? Lay::off(k + 1) : 0;
            const int cb = 1 + (k - 2) * P * P;
            // Suffix (exclusive, over j' > j) of the next level's row-adjoint
            // inputs, per r'.
            T Ab = (k < NL) ? Abar[on] : T(0);
#pragma unroll
            for (int rr = 1; rr < P; ++rr) Ub[rr] = T(0);
            if (k < NL) {
#pragma unroll
              for (int rr = 1; rr < P; ++rr) {
                if (rr < fn) {
                  T tu = T(0);
#pragma unroll
                  for (int c = 0; c < C; ++c)
                    tu += Z[c] * (T(1) / T(rr + 1)) * Rb_next[c][rr][0];
                  const T inc = warp_suffix_incl(tu, lane);
                  Ub[rr] = inc - tu + bcarry[on + rr];
                  if (lane == 0 && s > 0) BR[(long long)r * NX + on + rr] = inc + bcarry[on + rr];
                }
              }
            }
            // Right to left over the lane's cells.
#pragma unroll
            for (int c = C - 1; c >= 0; --c) {
              const T z = Z[c];
              T Rb[P][P];
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) {
                  T v = T(0);
                  if (i < f && j < f) {
                    v = w[k];
                    if (k < NL) {
                      v += Ab;
                      if (j + 1 < fn) v += DA[on + j + 1][c];
                      if (i + 1 < fn) v += Ub[i + 1];
                      if (i + 1 < fn && j + 1 < fn)
                        v += z * (T(1) / T((i + 2) * (j + 2))) * Rb_next[c][i + 1][j + 1];
                    }
                  }
                  Rb[i][j] = v;
                }
              // Zbar contribution: coefficient of z in each state.
              if (k == 1) {
                Zb[c] += Rb[0][0];
              } else {
#pragma unroll
                for (int i = 0; i < P; ++i)
#pragma unroll
                  for (int j = 0; j < P; ++j)
                    if (i < f && j < f) Zb[c] += Rb[i][j] * coef[c][cb + i * P + j];
              }
              // Advance the horizontal suffixes (exclusive -> include cell c).
              if (k < NL) {
                Ab += DA[on][c];
#pragma unroll
                for (int rr = 1; rr < P; ++rr)
                  if (rr < fn) Ub[rr] += z * (T(1) / T(rr + 1)) * Rb_next[c][rr][0];
              }
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) Rb_next[c][i][j] = Rb[i][j];
            }
            // Level k+1's increments can go in now that level k has used DA.
            if (k < NL) {
#pragma unroll
              for (int c = 0; c < C; ++c)
#pragma unroll
                for (int rr = 0; rr < P; ++rr)
                  if (rr < fn) DA[on + rr][c] += pendDA[rr][c];
            }
            if (k >= 2) {
#pragma unroll
              for (int c = 0; c < C; ++c) {
                pendDA[0][c] = Z[c] * Rb_next[c][0][0];
#pragma unroll
                for (int rr = 1; rr < P; ++rr)
                  pendDA[rr][c] = (rr < f) ? Z[c] * (T(1) / T(rr + 1)) * Rb_next[c][0][rr] : T(0);
              }
            }
          }
          // Cells outside the pair (padding, the next strip's cell) carry no
          // adjoint.
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const int j = g0 + c;
            if (r >= lx || j >= ly || (lane == 31 && c == C - 1)) Zb[c] = T(0);
          }
        } else {
#pragma unroll
          for (int c = 0; c < C; ++c) { Zb[c] = T(0); Mlo[c] = T(0); arglo[c] = T(0); }
        }
        // ---- Mbar on grid row r+1 and its pull-back ----
        const T zl_lo = shfl_up(Zb[C - 1], 1);
        const T zl_hi = shfl_up(Zbhi[C - 1], 1);
        T q[VP];
#pragma unroll
        for (int k = 0; k < VP; ++k) q[k] = T(0);
        T sw = T(0);
        const int gi = r + 1;  // grid row being finalised
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const T lo_l = (c == 0) ? (lane == 0 ? T(0) : zl_lo) : Zb[c - 1];
          const T hi_l = (c == 0) ? (lane == 0 ? T(0) : zl_hi) : Zbhi[c - 1];
          const T mbar = lo_l - Zb[c] - hi_l + Zbhi[c];
          const int j = g0 + c;
          const bool valid = j < Ly && gi < Lx;
          const T W = valid ? (rbf ? mbar * Mhi[c] : mbar) : T(0);
          sw += W;
#pragma unroll
          for (int k = 0; k < KD; ++k) q[k] = fma(W, yv[c][k], q[k]);
          if (valid) {
            // d/dparam: RBF M |x-y|^2 / s^3 with |x-y|^2 = -arg / alpha;
            // linear M / s.
            dpar += rbf ? (double)W * (-(double)arghi[c] / alpha) : (double)W * (double)Mhi[c];
          }
        }
        // dX row gi: RBF (1/s^2) sum_j W (y_j - x), linear s sum_j Mbar y_j.
        if (rbf) {
          const T inv2a = T(1) / T(2.0 * alpha);
#pragma unroll
          for (int k = 0; k < KD; ++k) q[k] -= sw * (xhi[k] * inv2a);
        }
        const T tot = transpose_reduce<T, VP>(q, lane);
        const int idx = red_index<VP>(lane);
        if ((lane & (32 / VP - 1)) == 0) {  // one lane per reduced value
          if (idx < args.d && gi < Lx) {
            const double scale = rbf ? 1.0 / (args.param * args.param) : args.param;
            T* dst = args.dX + ((long long)a * args.LX + gi) * args.d + idx;
            atomicAdd(dst, (T)(scale * (double)tot));
          }
        }
#pragma unroll
        for (int c = 0; c < C; ++c) { Mhi[c] = Mlo[c]; arghi[c] = arglo[c]; Zbhi[c] = Zb[c]; }
#pragma unroll
        for (int k = 0; k < RS; ++k) xhi[k] = xlo[k];
      }
      if (ns > 1) __syncwarp();
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
