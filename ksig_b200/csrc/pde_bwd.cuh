// Adjoint of the Goursat-PDE signature kernel (no reference counterpart: the
// reference has no gradients).
//
// Forward scheme per refined cell (ksig/algorithms.py:384-385, q = Z / F^2):
//   K[i+1,j+1] = A (K[i,j+1] + K[i+1,j]) - B K[i,j],
//   A = 1 + q/2 + q^2/12, B = 1 - q^2/12, output K[N, M].
// Exact discrete adjoint: with L = w K[N, M] and G(i,j) = dL/dK[i+1,j+1]
// (the adjoint of a refined cell's lower-right corner),
//   G(i,j) = A(i+1,j) G(i+1,j) + A(i,j+1) G(i,j+1) - B(i+1,j+1) G(i+1,j+1)
// (cells outside the grid contribute nothing), seeded by G(N-1,M-1) = w, and
//   dL/dq(i,j) = G(i,j) ((K[i,j+1] + K[i+1,j]) (1/2 + q/6) + K[i,j] q/6).
// Rows are swept bottom-up and columns right to left in increment form:
// with H(i,j) = G(i,j) - G(i+1,j),
//   H(i,j) = H(i,j+1) + (A(i+1,j)-1) G(i+1,j) + (A(i,j+1)-1) G(i,j+1)
//            + (1-B(i+1,j+1)) G(i+1,j+1),
// which keeps FP32 rounding small, as the forward's increment form does.
// The seed enters as H(N-1, M) = w.
//
// One warp per pair; lane l owns C cell columns (C*F refined columns) of a
// strip of 32*C-1 cells, as in the forward sweep.
// Phase 1 is the forward sweep (lane l one row behind lane l-1).  Per step
// every lane records only the boundary of its block of the K grid: the
// bottom refined row (C*F values) and the K and H values it received from
// the left (2F values), in a lane-minor layout [step][value][lane], so the
// stores of a warp are contiguous.
// Phase 2 is its exact time reversal: lane l is one row behind lane l+1, so
// the adjoint's row increments H, the G values at the lane boundary and the
// neighbouring cell's q arrive from lane l+1 by __shfl_down.  Every lane
// reads the record slots of the same step (contiguous loads), rebuilds the
// F x C*F interior of its K block with the forward's own arithmetic (so the
// values are the forward's, bit for bit) into shared memory, and runs the
// adjoint over it.
// It forms dL/dZ per cell and pulls it back through the second difference
// and the static kernel into dX and dparam like the DP adjoint: lane l
// covers its C grid columns plus the next lane's first one, and the dX
// vector of a grid row is summed along the lanes and added once per row
// and strip.
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
  T* scratch;             // per warp, see pde_bwd_scratch_elems
  long long scratch_per_warp;
  int ns_max, rows_max;
  int* status;
};

// Scratch elements per warp:
//   REC [ns_max][rows_max + 32][C*F + 2F][32]  boundary records of phase 1
//   BL  [2][rows_max][2F]                       forward strip carries
//   BR  [2][rows_max][2F + 1]                   adjoint strip carries
__host__ __device__ inline long long pde_bwd_scratch_elems(int ns_max, int rows_max, int c,
                                                           int f) {
  return (long long)ns_max * (rows_max + 32) * (c * f + 2 * f) * 32 +
         2LL * rows_max * 2 * f + 2LL * rows_max * (2 * f + 1);
}

// Dynamic shared memory per block: the rebuilt K block of each lane,
// [F][C*F + 1][32] per warp.
__host__ __device__ inline size_t pde_bwd_smem_bytes(int wpb, int c, int f, size_t es) {
  return (size_t)wpb * f * (c * f + 1) * 32 * es;
}

template <typename T, int KD, int C, int F, int WPB>
__global__ void __launch_bounds__(WPB * 32)
pde_bwd_kernel(const PdeBwdArgs<T> args) {
  constexpr int RS = packed_stride<T>(KD);
  constexpr int VN = Vec<T>::N;
  using V = typename Vec<T>::type;
  constexpr int STRIP = 32 * C - 1;
  constexpr int CF = C * F;
  constexpr int RW = CF + 1;      // K row of a block: CF refined columns + the left column
  constexpr int RR = CF + 2 * F;  // record: bottom K row, left K and H per refined row
  constexpr int NB = 2 * F + 1;   // adjoint carry: H and G per refined row, q of the cell
  constexpr T invF2 = T(1) / T(F * F);

  extern __shared__ __align__(16) unsigned char dsm[];
  const int lane = threadIdx.x & 31;
  T* ks = reinterpret_cast<T*>(dsm) + (size_t)(threadIdx.x >> 5) * F * RW * 32 + lane;
  const long long wg = (long long)blockIdx.x * WPB + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * WPB;
  T* scr = args.scratch + wg * args.scratch_per_warp;
  const long long steps = (long long)args.rows_max + 32;
  const long long rm = args.rows_max;
  T* REC = scr;
  T* BL = REC + (long long)args.ns_max * steps * RR * 32;
  T* BR = BL + 2 * rm * 2 * F;
  auto rec_at = [&](int s, long long t) {
    return REC + ((long long)s * steps + t) * RR * 32 + lane;
  };

  const double alpha = 1.4426950408889634 / fmax(2.0 * args.param * args.param, 1e-12);
  const bool rbf = args.kind == KIND_RBF;
  const bool want_dpar = args.dparam != nullptr;
  const T ralpha = T(alpha);
  // dM/dx = M (y - x) / s^2 (RBF; the row sums below carry 2a (y - x)) or
  // s y (linear).
  const double xscale =
      rbf ? 1.0 / (args.param * args.param) / (2.0 * alpha) : args.param;
  double dpar_w = 0.0;

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
    if (ns > args.ns_max || lx > args.rows_max) {
      if (lane == 0) set_status(args.status, KSIG_ERR_DEVICE);
      continue;
    }
    const T w = (T)args.grad[task];
    const T* xb = args.xr + args.xstart[a] * RS;
    const T* yb = args.yr + args.ystart[b] * RS;

    // The lane's C+1 grid columns of strip s.
    T yv[C + 1][KD + 1];
    auto load_y = [&](int s) {
#pragma unroll
      for (int c = 0; c <= C; ++c) {
        int col = s * STRIP + C * lane + c;
        col = col < Ly - 1 ? col : Ly - 1;
        const V* p = reinterpret_cast<const V*>(yb + (long long)col * RS);
        T tmp[RS];
#pragma unroll
        for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(tmp)[v] = __ldg(p + v);
#pragma unroll
        for (int k = 0; k <= KD; ++k) yv[c][k] = tmp[k];
      }
      // RBF: the lane-centred frame of rbf_center_cols.
      if (rbf) rbf_center_cols<KD, C + 1>(yv, ralpha);
    };
    auto gram = [&](int row, T (&m)[C + 1], T (&arg)[C + 1]) {
      row = row < 0 ? 0 : (row > lx ? lx : row);
      const V* p = reinterpret_cast<const V*>(xb + (long long)row * RS);
      T xv[RS];
#pragma unroll
      for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(p + v);
      if (rbf) {
        T xt[RS];
        rbf_center_row<KD>(xv, yv[0], ralpha, xt);
        arg[0] = xt[KD];
        m[0] = kexp2(xt[KD]);
#pragma unroll
        for (int c = 1; c <= C; ++c) {
          arg[c] = centred_arg<KD, false>(xt, yv[c], xt[KD]);
          m[c] = kexp2(arg[c]);
        }
      } else {
#pragma unroll
        for (int c = 0; c <= C; ++c) {
          arg[c] = packed_arg<KD, false>(xv, yv[c], T(0));
          m[c] = arg[c];
        }
      }
    };

    // ------------- phase 1: forward, top-down, strips left to right --------
    for (int s = 0; s < ns; ++s) {
      load_y(s);
      const int g0 = s * STRIP + C * lane;
      const T* blin = BL + (long long)((s + 1) & 1) * rm * 2 * F;  // from strip s - 1
      T* blout = BL + (long long)(s & 1) * rm * 2 * F;
      T Mlo[C + 1], Mhi[C + 1], argd[C + 1];
      gram(0, Mlo, argd);
      T Kr[CF];
#pragma unroll
      for (int j = 0; j < CF; ++j) Kr[j] = T(1);
      T kcorner = T(1);
      T X[2 * F];  // outgoing: K of the last refined column, H, per refined row
#pragma unroll
      for (int h = 0; h < 2 * F; ++h) X[h] = T(0);
      for (int t = 0; t < lx + 32; ++t) {
        const int r = t - lane;
        T Xin[2 * F];
#pragma unroll
        for (int h = 0; h < 2 * F; ++h) Xin[h] = shfl_up(X[h], 1);
        if (r >= 0 && r < lx) {
          gram(r + 1, Mhi, argd);
          if (lane == 0) {
            if (s > 0) {
#pragma unroll
              for (int h = 0; h < 2 * F; ++h) Xin[h] = __ldcg(blin + (long long)r * 2 * F + h);
            } else {
#pragma unroll
              for (int f = 0; f < F; ++f) { Xin[f] = T(1); Xin[F + f] = T(0); }
            }
          }
          T a_[C], b_[C];
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const bool valid = g0 + c < ly && !(lane == 31 && c == C - 1);
            const T z = valid ? (Mhi[c + 1] - Mhi[c] - Mlo[c + 1] + Mlo[c]) : T(0);
            const T q = z * invF2;
            b_[c] = q * q * (T(1) / T(12));
            a_[c] = fma(T(0.5), q, b_[c]);
          }
          T* rp = rec_at(s, t);
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
                const int J = c * F + g;
                const T kro = Kr[J];
                const T gg = fma(kro + kln, a_[c], klo * b_[c]);
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
          }
          // Record the block's boundary: its bottom K row and what came in
          // from the left.
#pragma unroll
          for (int j = 0; j < CF; ++j) rp[j * 32] = Kr[j];
#pragma unroll
          for (int h = 0; h < 2 * F; ++h) rp[(CF + h) * 32] = Xin[h];
          kcorner = Xin[F - 1];
          if (lane == 31 && s + 1 < ns) {
#pragma unroll
            for (int h = 0; h < 2 * F; ++h) __stcg(blout + (long long)r * 2 * F + h, X[h]);
          }
#pragma unroll
          for (int c = 0; c <= C; ++c) Mlo[c] = Mhi[c];
        }
      }
      __syncwarp();  // carries and records of this strip -> later readers
    }

    // ------------- phase 2: adjoint, bottom-up, strips right to left -------
    for (int s = ns - 1; s >= 0; --s) {
      load_y(s);
      const int g0 = s * STRIP + C * lane;
      const T* brin = BR + (long long)((s + 1) & 1) * rm * NB;  // from strip s + 1
      T* brout = BR + (long long)(s & 1) * rm * NB;
      T Mprev[C + 1], argprev[C + 1];
#pragma unroll
      for (int c = 0; c <= C; ++c) { Mprev[c] = T(0); argprev[c] = T(0); }
      T Zprev[C], Zbprev[C];
#pragma unroll
      for (int c = 0; c < C; ++c) { Zprev[c] = T(0); Zbprev[c] = T(0); }
      T Gb[CF];  // G of the refined row below the current cell row
#pragma unroll
      for (int j = 0; j < CF; ++j) Gb[j] = T(0);
      T Aprev[NB];
#pragma unroll
      for (int h = 0; h < NB; ++h) Aprev[h] = T(0);
      T accprev[KD];
#pragma unroll
      for (int k = 0; k < KD; ++k) accprev[k] = T(0);
      T gr_below = T(0), zr_below = T(0);  // lane l+1's G and q one cell row down
      for (int u = 0; u < lx + 33; ++u) {
        const int rho = u - (31 - lane);
        const int r = lx - rho;                      // cell row; grid row computed
        const bool act = rho >= 1 && rho <= lx;      // cell row r exists
        const bool fin = rho >= 1 && rho <= lx + 1;  // grid row r + 1 completes here
        T Ain[NB];
#pragma unroll
        for (int h = 0; h < NB; ++h) Ain[h] = shfl_down(Aprev[h], 1);
        T acc[KD];
#pragma unroll
        for (int k = 0; k < KD; ++k) acc[k] = shfl_down(accprev[k], 1);
        if (lane == 31) {
#pragma unroll
          for (int k = 0; k < KD; ++k) acc[k] = T(0);
#pragma unroll
          for (int h = 0; h < NB; ++h)
            Ain[h] = (s + 1 < ns && act) ? __ldcg(brin + (long long)r * NB + h) : T(0);
          if (s + 1 == ns && act && r == lx - 1) Ain[F - 1] = w;  // seed H(N-1, M) = w
        }
        T Mnew[C + 1], argn[C + 1];
        gram(r, Mnew, argn);
        T Z[C], Zb[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const bool valid = act && g0 + c < ly && !(lane == 31 && c == C - 1);
          Z[c] = valid ? (Mprev[c + 1] - Mprev[c] - Mnew[c + 1] + Mnew[c]) : T(0);
          Zb[c] = T(0);
        }
        T Aout[NB];
#pragma unroll
        for (int h = 0; h < NB; ++h) Aout[h] = T(0);
        if (act) {
          const long long t = (long long)lx + 31 - u;  // phase-1 step of this cell row
          const T* rb = rec_at(s, t);
          // K row above the block: the bottom row of the cell row above
          // (its left corner is the left K of that row's last refined row),
          // or the boundary value 1.
          T top[RW];
          if (r > 0) {
            const T* ra = rec_at(s, t - 1);
#pragma unroll
            for (int j = 0; j < CF; ++j) top[j] = ra[j * 32];
            top[CF] = ra[(CF + F - 1) * 32];
          } else {
#pragma unroll
            for (int j = 0; j < RW; ++j) top[j] = T(1);
          }
          // Rebuild the block's K rows with the forward's arithmetic.
          {
            T a_[C], b_[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const T q = Z[c] * invF2;
              b_[c] = q * q * (T(1) / T(12));
              a_[c] = fma(T(0.5), q, b_[c]);
            }
            T Kr[CF];
#pragma unroll
            for (int j = 0; j < CF; ++j) Kr[j] = top[j];
#pragma unroll
            for (int f = 0; f < F; ++f) {
              const T kin = rb[(CF + f) * 32];
              T klo = (f == 0) ? top[CF] : rb[(CF + (f > 0 ? f - 1 : 0)) * 32];
              T kln = kin;
              T H = rb[(CF + F + f) * 32];
#pragma unroll
              for (int c = 0; c < C; ++c) {
                const bool skip = (c == C - 1) && lane == 31;
#pragma unroll
                for (int g = 0; g < F; ++g) {
                  const int J = c * F + g;
                  const T kro = Kr[J];
                  const T gg = fma(kro + kln, a_[c], klo * b_[c]);
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
#pragma unroll
              for (int j = 0; j < CF; ++j) ks[(f * RW + j) * 32] = Kr[j];
              ks[(f * RW + CF) * 32] = kin;
            }
          }
          T Kbot[RW], Ktop[RW];
#pragma unroll
          for (int j = 0; j < RW; ++j) Kbot[j] = ks[((F - 1) * RW + j) * 32];
          T Gbel[CF], Gcur[CF];
#pragma unroll
          for (int j = 0; j < CF; ++j) { Gbel[j] = Gb[j]; Gcur[j] = T(0); }
#pragma unroll
          for (int f = F - 1; f >= 0; --f) {
            if (f > 0) {
#pragma unroll
              for (int j = 0; j < RW; ++j) Ktop[j] = ks[((f > 0 ? f - 1 : 0) * RW + j) * 32];
            } else {
#pragma unroll
              for (int j = 0; j < RW; ++j) Ktop[j] = top[j];
            }
            const bool last_f = f == F - 1;
            T H = Ain[f];
            T Gr = Ain[F + f];
            T Gbr = last_f ? gr_below : Ain[F + (f + 1 < F ? f + 1 : 0)];
            T qr_cell = Ain[2 * F] * invF2;
            T qo_cell = last_f ? zr_below * invF2 : qr_cell;
#pragma unroll
            for (int c = C - 1; c >= 0; --c) {
              const bool skip = (c == C - 1) && lane == 31;
              const T qown = Z[c] * invF2;
              const T qb = last_f ? Zprev[c] * invF2 : qown;
              const T abq = qb * fma(qb, T(1) / T(12), T(0.5));
              const T q6 = qown * (T(1) / T(6));
              T zb = T(0);
#pragma unroll
              for (int g = F - 1; g >= 0; --g) {
                const int J = c * F + g;
                const T qr = (g < F - 1) ? qown : qr_cell;
                const T qo = (g < F - 1) ? qb : qo_cell;
                const T arq = qr * fma(qr, T(1) / T(12), T(0.5));
                const T boq = qo * qo * (T(1) / T(12));
                const T Gbelow = Gbel[J];
                const T Hn = fma(abq, Gbelow, fma(arq, Gr, fma(boq, Gbr, H)));
                const T G = Gbelow + Hn;
                const T Ktr = Ktop[J];
                const T Ktl = J > 0 ? Ktop[J > 0 ? J - 1 : 0] : Ktop[CF];
                const T Kbl = J > 0 ? Kbot[J > 0 ? J - 1 : 0] : Kbot[CF];
                const T dq = G * fma(Ktr + Kbl, T(0.5) + q6, Ktl * q6);
                if (!skip) {
                  H = Hn;
                  Gr = G;
                  Gbr = Gbelow;
                  Gcur[J] = G;
                  zb += dq;
                }
              }
              Zb[c] += zb;
              if (!skip) {
                qr_cell = qown;
                qo_cell = qb;
              }
            }
            Aout[f] = H;
            Aout[F + f] = Gr;
#pragma unroll
            for (int j = 0; j < CF; ++j) Gbel[j] = Gcur[j];
#pragma unroll
            for (int j = 0; j < RW; ++j) Kbot[j] = Ktop[j];
          }
          Aout[2 * F] = Z[0];
#pragma unroll
          for (int j = 0; j < CF; ++j) Gb[j] = Gbel[j];
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const bool valid = g0 + c < ly && !(lane == 31 && c == C - 1);
            Zb[c] = valid ? Zb[c] * invF2 : T(0);
          }
          if (lane == 0 && s > 0) {
#pragma unroll
            for (int h = 0; h < NB; ++h) __stcg(brout + (long long)r * NB + h, Aout[h]);
          }
        }

        // ---- grid row p = r + 1: partial Mbar of this lane's cells ----
        const int p = r + 1;
        T dp = T(0), sw = T(0);
#pragma unroll
        for (int c = 0; c <= C; ++c) {
          T mb = (c < C) ? Zbprev[c < C ? c : 0] - Zb[c < C ? c : 0] : T(0);
          if (c > 0) mb += Zb[c - 1] - Zbprev[c - 1];
          const int q = g0 + c;
          const bool valid = fin && q < Ly && (c < C || lane < 31);
          const T W = valid ? (rbf ? mb * Mprev[c] : mb) : T(0);
          // RBF: column 0 is the lane's centre (y' = 0); the other columns
          // hold 2a y' in the lane's frame.
          if (!rbf || c > 0) {
#pragma unroll
            for (int k = 0; k < KD; ++k) acc[k] = fma(W, yv[c][k], acc[k]);
          }
          sw += W;
          dp = fma(W, rbf ? argprev[c] : Mprev[c], dp);
        }
        if (want_dpar) dpar_w += (double)dp;
        if (rbf) {
          // 2a sum_c W_c (y_c - x_p) = sum_c W_c 2a y'_c - 2a x'_p sum_c W_c:
          // frame-independent, so the lanes' shares add up along the row.
          const V* xp = reinterpret_cast<const V*>(xb + (long long)(p < 0 ? 0 : (p < lx ? p : lx)) * RS);
          T xv[RS];
#pragma unroll
          for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(xp + v);
          const T t = T(-2) * ralpha * sw;
#pragma unroll
          for (int k = 0; k < KD; ++k) acc[k] = fma(xv[k] + yv[0][k], t, acc[k]);
        }
        if (lane == 0 && fin) {
          T* dst = args.dX + ((long long)a * args.LX + p) * args.d;
#pragma unroll
          for (int k = 0; k < KD; ++k) {
            if (k < args.d) atomicAdd(dst + k, (T)(xscale * (double)acc[k]));
          }
        }
#pragma unroll
        for (int k = 0; k < KD; ++k) accprev[k] = acc[k];
        gr_below = Ain[F];
        zr_below = Ain[2 * F];
#pragma unroll
        for (int h = 0; h < NB; ++h) Aprev[h] = Aout[h];
#pragma unroll
        for (int c = 0; c < C; ++c) { Zprev[c] = Z[c]; Zbprev[c] = Zb[c]; }
#pragma unroll
        for (int c = 0; c <= C; ++c) { Mprev[c] = Mnew[c]; argprev[c] = argn[c]; }
      }
      __syncwarp();  // adjoint carries of this strip -> the next strip
    }
  }
  if (want_dpar) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dpar_w += __shfl_xor_sync(FULL, dpar_w, o);
    if (lane == 0 && dpar_w != 0.0) {
      const double p = args.param;
      atomicAdd(args.dparam, rbf ? -dpar_w / (alpha * p * p * p) : dpar_w / p);
    }
  }
}

}  // namespace ksig
