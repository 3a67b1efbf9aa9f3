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
// One warp per pair, skewed like the forward sweep: lane l owns C adjacent
// columns of a strip of 32*C-1 cells.
//
// Phase 1 runs the forward top-down with lane l one row behind lane l-1
// (horizontal prefixes handed on by __shfl_up).  Every lane records, per
// step, the horizontal prefixes it received (coalesced, [step][h][lane]);
// the final column sums stay in registers (last strip) or go to scratch.
//
// Phase 2 is the exact time reversal of phase 1: lane l is now one row
// behind lane l+1.  Per cell row it
//   - recovers the forward state at the row by subtracting the row's
//     contributions from the column sums, with the left-boundary prefixes
//     read back from the record (no per-cell activations are stored);
//   - forms the adjoint: column suffix sums stay in the lane's registers,
//     horizontal suffixes arrive from lane l+1 by __shfl_down;
//   - pulls Zbar back to Mbar and into dX for the grid row it completes.
//     Lane l covers its C grid columns plus the next lane's first one
//     (partial Mbar from its own cells); the per-row dX vector is summed
//     along the lanes by __shfl_down and added once per row and strip.
// Order 1 takes one left-to-right pass per row (the horizontal suffix of a
// row is the lane total minus a running prefix); order p >= 2 keeps each
// cell's horizontal prefixes left to right and runs the adjoint right to
// left, rebuilding the cell coefficients from them.
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
  const int* order;      // optional task permutation (longest first)
  int ntasks, nX, nYseq;
  int kind;
  double param;
  const double* glev;    // [nl_out + 1, ntasks] dL/dlevel (row 0 unused)
  int nl_out;
  T* dX;                 // [nX, LX, d] row-side gradient (accumulated)
  int LX, d;
  double* dparam;        // scalar (accumulated), may be null
  T* scratch;            // per warp, see dp_bwd_scratch_elems
  long long scratch_per_warp;
  int ns_max, rows_max;
  int* status;
  // Split gradient pass (order 1): phases 1 = forward pass only, writing the
  // level totals to `lev` ([nl_out + 1, ntasks]); 2 = adjoint pass only,
  // replaying the records a phase-1 launch left in `rec`; 0 or 3 = both in
  // one launch.  `rec`: records per pair (rec_per_pair elements each) instead
  // of per warp.
  int phases;
  // Strip checkpointing (one-launch adjoint of multi-strip pairs): phase 1
  // keeps every strip's left-boundary stream and final column sums but the
  // per-step records of the last strip only; phase 2 recomputes each other
  // strip's records from its checkpoint just before its adjoint.  The
  // records then need one strip of scratch instead of ns_max.
  int ckpt;
  T* rec;
  long long rec_per_pair;
  double* lev;
};

// Scratch elements per warp:
//   REC [ns_max][rows_max + 33][NX][32]  phase-1 incoming prefixes per step
//                                        ([1][...] with strip checkpointing)
//   CS  [ns_max][NX][C][32]              final column sums per strip
//   BL  [2][rows_max][NX]                forward strip-to-strip carries
//                                        ([ns_max][...] with checkpointing)
//   BR  [2][rows_max][NX]                adjoint strip-to-strip carries
__host__ __device__ inline long long dp_bwd_scratch_elems(int ns_max, int rows_max, int nx,
                                                          int c, int ckpt = 0) {
  return (long long)(ckpt ? 1 : ns_max) * (rows_max + 33) * nx * 32 +
         (long long)ns_max * nx * c * 32 + (long long)(ckpt ? ns_max + 2 : 4) * rows_max * nx;
}

// Dynamic shared memory per block: each lane keeps its C + 1 packed column
// points of the current strip in shared memory ([C+1][RV][32] 16-byte
// vectors per warp) instead of registers.
__host__ __device__ inline size_t dp_bwd_smem_bytes(int wpb, int c, int rs, size_t es) {
  return (size_t)wpb * (c + 1) * (rs * es / 16) * 32 * 16;
}

// Kernel body.  RBF_NOPAR: RBF static kernel and no parameter gradient,
// known at compile time (no per-point kind tests, no distance arguments
// kept for dparam).
template <typename T, int KD, int C, int NL, int P, int WPB, bool RBF_NOPAR, bool FWD_ONLY,
          bool CKPT = false>
__device__ __forceinline__ void dp_bwd_body(const DpBwdArgs<T>& args) {
  using Lay = DpLayout<NL, P>;
  constexpr int NH = Lay::NH;
  constexpr int NX = NH > 0 ? NH : 1;
  constexpr int RS = packed_stride<T>(KD);
  constexpr int VN = Vec<T>::N;
  constexpr int RV = RS / VN;
  using V = typename Vec<T>::type;
  constexpr int STRIP = 32 * C - 1;
  // Two steps per loop trip remove the per-step register moves of the
  // pipelined row state.  FP32 order 1 only: the order >= 2 and FP64
  // instances hold more state per cell, and there the unrolled loop spills
  // more and runs slower.  The adjoint pass (phase 2) of the 7-column tiles
  // runs one step per trip since the lane-centred Gram raised its state:
  // unrolled it spilled 920 bytes at d = 9, and one step per trip took the
  // 512 x 512 adjoint from 86.5 to 78 ms on B200.  Phase 1 keeps two steps
  // per trip (one step: one-launch adjoint 78 -> 82 ms, forward-only pass
  // 23 -> 35 ms).
  constexpr int kStepUnroll = (sizeof(T) == 4 && P == 1) ? 2 : 1;
  constexpr int kStepUnroll2 = (sizeof(T) == 4 && P == 1 && C < 7) ? 2 : 1;
  // Paired FP32 Gram arguments (packed_arg) where they keep the occupancy.
  constexpr bool kPairArg = sizeof(T) == 4 && KD <= 16 && (C >= 7 || P >= 2);

  extern __shared__ __align__(16) unsigned char dsm[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  V* ysm = reinterpret_cast<V*>(dsm) + (size_t)wib * (C + 1) * RV * 32;
  const long long wg = (long long)blockIdx.x * WPB + wib;
  const long long nw = (long long)gridDim.x * WPB;
  T* scr = args.scratch + wg * args.scratch_per_warp;
  const long long steps_max = (long long)args.rows_max + 33;
  const long long rm = args.rows_max;
  // Strip checkpointing is compiled into its own kernel (dp_bwd_ckpt_kernel),
  // so that the recompute path does not weigh on the others' registers.
  constexpr bool ckpt = CKPT;
  const long long cs_off = (long long)(ckpt ? 1 : args.ns_max) * steps_max * NX * 32;
  T* const REC0 = scr;
  T* BL = REC0 + cs_off + (long long)args.ns_max * NX * C * 32;
  T* BR = BL + (long long)(ckpt ? args.ns_max : 2) * rm * NX;
  const int phases = FWD_ONLY ? 1 : (args.phases ? args.phases : 3);

  const double alpha = 1.4426950408889634 / fmax(2.0 * args.param * args.param, 1e-12);
  const bool rbf = RBF_NOPAR || args.kind == KIND_RBF;
  const bool want_dpar = !RBF_NOPAR && args.dparam != nullptr;
  const T ralpha = T(alpha);
  // dM/dx = M (y - x) / s^2 (RBF; the row sums below carry 2a (y - x)) or
  // s y (linear).
  const double xscale = rbf ? 1.0 / (args.param * args.param) : args.param;
  const T xscale_t = T(rbf ? xscale / (2.0 * alpha) : xscale);
  double dpar_w = 0.0;

  for (long long tid = wg; tid < args.ntasks; tid += nw) {
    const int2 ab = decode_task((int)tid, args.mode, args.nY, args.list, args.order);
    const int task = args.order ? args.order[tid] : (int)tid;
    T* REC = args.rec ? args.rec + (long long)task * args.rec_per_pair : REC0;
    T* CS = REC + cs_off;
    if constexpr (FWD_ONLY) {
      if (lane == 0) args.lev[task] = 1.0;  // level 0; levels >= 1 start at 0
    }
    if (ab.x < 0 || ab.x >= args.nX || ab.y < 0 || ab.y >= args.nYseq) {
      if (lane == 0) set_status(args.status, KSIG_ERR_INVALID);
      continue;
    }
    const int a = ab.x, b = ab.y;
    const int Lx = args.xlen[a], Ly = args.ylen[b];
    const int lx = Lx - 1, ly = Ly - 1;
    if (lx <= 0 || ly <= 0) continue;  // no cells: levels >= 1 are constant
    const int ns = (ly + STRIP - 1) / STRIP;
    if (ns > args.ns_max || lx > args.rows_max) {
      if (lane == 0) set_status(args.status, KSIG_ERR_DEVICE);
      continue;
    }
    T w[NL + 1];
#pragma unroll
    for (int k = 0; k <= NL; ++k)
      w[k] = (!FWD_ONLY && k >= 1 && k <= args.nl_out)
                 ? (T)args.glev[(long long)k * args.ntasks + task] : T(0);

    const T* xb = args.xr + args.xstart[a] * RS;
    const T* yb = args.yr + args.ystart[b] * RS;
    // Column points of strip s (C own columns + the next lane's first).
    // RBF: stored in the lane-centred frame of rbf_center_cols (slot 0 the
    // negated centre, slots 1..C relative to it).
    auto stage_y = [&](int s) {
      const int col0 = s * STRIP + C * lane;
      T c0[RS];
      {
        const V* p = reinterpret_cast<const V*>(yb + (long long)(col0 < Ly - 1 ? col0 : Ly - 1) * RS);
#pragma unroll
        for (int v = 0; v < RV; ++v) reinterpret_cast<V*>(c0)[v] = __ldg(p + v);
      }
#pragma unroll
      for (int c = 1; c <= C; ++c) {
        int col = col0 + c;
        col = col < Ly - 1 ? col : Ly - 1;
        const V* p = reinterpret_cast<const V*>(yb + (long long)col * RS);
        T yv[RS];
#pragma unroll
        for (int v = 0; v < RV; ++v) reinterpret_cast<V*>(yv)[v] = __ldg(p + v);
        if (rbf) rbf_center_col<KD>(yv, c0, ralpha);
#pragma unroll
        for (int v = 0; v < RV; ++v) ysm[(c * RV + v) * 32 + lane] = reinterpret_cast<V*>(yv)[v];
      }
      if (rbf) {
#pragma unroll
        for (int k = 0; k < KD; ++k) c0[k] = -c0[k];
      }
#pragma unroll
      for (int v = 0; v < RV; ++v) ysm[v * 32 + lane] = reinterpret_cast<V*>(c0)[v];
    };
    auto y_col = [&](int c, T (&yv)[RS]) {
#pragma unroll
      for (int v = 0; v < RV; ++v) reinterpret_cast<V*>(yv)[v] = ysm[(c * RV + v) * 32 + lane];
    };
    auto load_x = [&](int row, T (&xv)[RS]) {
      row = row < 0 ? 0 : (row > lx ? lx : row);
      const V* p = reinterpret_cast<const V*>(xb + (long long)row * RS);
#pragma unroll
      for (int v = 0; v < RV; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(p + v);
    };
    auto gram_row = [&](const T (&xv)[RS], T (&m)[C], T (&arg)[C]) {
      if (rbf) {
        T negc[RS], xt[RS];
        y_col(0, negc);
        rbf_center_row<KD>(xv, negc, ralpha, xt);
        arg[0] = xt[KD];
        m[0] = kexp2(xt[KD]);
#pragma unroll
        for (int c = 1; c < C; ++c) {
          T yv[RS];
          y_col(c, yv);
          const T acc = centred_arg<KD, kPairArg>(xt, yv, xt[KD]);
          arg[c] = acc;
          m[c] = kexp2(acc);
        }
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) {
          T yv[RS];
          y_col(c, yv);
          const T acc = packed_arg<KD, kPairArg>(xv, yv, T(0));
          arg[c] = acc;
          m[c] = acc;
        }
      }
    };
    auto rec_at = [&](int s, long long t) {
      return REC + ((long long)(ckpt ? 0 : s) * steps_max + t) * NX * 32;
    };
    // Forward carries of strip s (its lane 31's exchange values per row).
    auto bl_at = [&](int s) { return BL + (long long)(ckpt ? s : (s & 1)) * rm * NX; };

    T Ccol[NX][C];  // forward column sums (rows above the current row)
    // Forward-only launches: per-lane level totals (FP64), levels 1..NL.
    double lt[NL + 1];
#pragma unroll
    for (int k = 0; k <= NL; ++k) lt[k] = 0.0;

    // ---------------- phase 1: forward, top-down, strips left to right -----
    // One strip of the forward pass: records (rec_on), carries to the next
    // strip and final column sums (cs_on).  Phase 2 calls it again for the
    // strips whose records were not kept (strip checkpointing).
    auto fwd_strip = [&](int s, bool rec_on, bool cs_on) {
      stage_y(s);
#pragma unroll
      for (int h = 0; h < NX; ++h)
#pragma unroll
        for (int c = 0; c < C; ++c) Ccol[h][c] = T(0);
      T Xout[NX];
#pragma unroll
      for (int h = 0; h < NX; ++h) Xout[h] = T(0);
      T Mprev[C], DMold[C];
#pragma unroll
      for (int c = 0; c < C; ++c) { Mprev[c] = T(0); DMold[c] = T(0); }
      T xc[RS];
      load_x(-lane, xc);
      const T* blin = bl_at(s > 0 ? s - 1 : 1);  // written by strip s - 1 (read when s > 0)
      T* blout = bl_at(s);
      const int T1 = lx + 33;
#pragma unroll kStepUnroll
      for (int t = 0; t < T1; ++t) {
        const int rho = t - lane;     // grid row computed this step
        const int r = rho - 2;        // cell row processed this step
        const bool act = r >= 0 && r < lx;
        T xn[RS];
        load_x(rho + 1, xn);
        T Mnew[C], argn[C];
        gram_row(xc, Mnew, argn);
        T DMnew[C];
#pragma unroll
        for (int c = 0; c < C; ++c) DMnew[c] = Mnew[c] - Mprev[c];
        // Lane l+1 has just formed the vertical difference of cell row r.
        const T right = shfl_down(DMnew[0], 1);
        T Xin[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h) Xin[h] = shfl_up(Xout[h], 1);
        if (lane == 0) {
#pragma unroll
          for (int h = 0; h < NX; ++h) Xin[h] = (s > 0 && act) ? blin[(long long)r * NX + h] : T(0);
        }
        T Z[C];
#pragma unroll
        for (int c = 0; c < C - 1; ++c) Z[c] = DMold[c + 1] - DMold[c];
        Z[C - 1] = lane == 31 ? T(0) : right - DMold[C - 1];
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (!act || s * STRIP + C * lane + c >= ly) Z[c] = T(0);
        if (rec_on && act && NH > 0) {
          T* rp = rec_at(s, t);
#pragma unroll
          for (int h = 0; h < NX; ++h) rp[h * 32 + lane] = Xin[h];
        }
        // Forward cell recursion (same arithmetic as DpPolicy::row).
        T H[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h) H[h] = Xin[h];
        if (P == 1) {
          T top = T(0);  // forward-only: this row's level-NL terms
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const T z = Z[c];
            T Hold[NX];
#pragma unroll
            for (int k = 2; k <= NL; ++k) {
              Hold[k - 2] = H[k - 2];
              H[k - 2] += Ccol[k - 2][c];
            }
            if (NL >= 2) Ccol[0][c] += z;
#pragma unroll
            for (int k = 2; k < NL; ++k) Ccol[k - 1][c] = fma(z, Hold[k - 2], Ccol[k - 1][c]);
            if constexpr (FWD_ONLY && NL >= 2) top = fma(z, Hold[NL - 2], top);
          }
          if constexpr (FWD_ONLY) lt[NL] += (double)top;
        } else {
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const T z = Z[c];
            T Rp[P][P];
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
              for (int j = 0; j < P; ++j) Rp[i][j] = T(0);
            Rp[0][0] = z;
            T tot = z;
#pragma unroll
            for (int k = 2; k <= NL; ++k) {
              const int f = Lay::f(k), fp = Lay::f(k - 1), o = Lay::off(k);
              T Rn[P][P];
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) Rn[i][j] = T(0);
              Rn[0][0] = z * H[o];
              H[o] += Ccol[o][c];
              Ccol[o][c] += tot;
              T lsum = Rn[0][0];
#pragma unroll
              for (int rr = 1; rr < P; ++rr) {
                if (rr < f) {
                  T Vs = T(0), Us = T(0);
#pragma unroll
                  for (int i = 0; i < P; ++i)
                    if (i < fp) { Vs += Rp[i][rr - 1]; Us += Rp[rr - 1][i]; }
                  const T zr = z * (T(1) / T(rr + 1));
                  Rn[0][rr] = zr * Ccol[o + rr][c];
                  Ccol[o + rr][c] += Vs;
                  Rn[rr][0] = zr * H[o + rr];
                  H[o + rr] += Us;
                  lsum += Rn[0][rr] + Rn[rr][0];
#pragma unroll
                  for (int ss = 1; ss < P; ++ss) {
                    if (ss < f) {
                      Rn[rr][ss] = z * (T(1) / T((rr + 1) * (ss + 1))) * Rp[rr - 1][ss - 1];
                      lsum += Rn[rr][ss];
                    }
                  }
                }
              }
              tot = lsum;
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) Rp[i][j] = Rn[i][j];
            }
          }
        }
#pragma unroll
        for (int h = 0; h < NX; ++h) Xout[h] = H[h];
        if (lane == 31 && act && s + 1 < ns) {
#pragma unroll
          for (int h = 0; h < NX; ++h) blout[(long long)r * NX + h] = Xout[h];
        }
#pragma unroll
        for (int c = 0; c < C; ++c) { Mprev[c] = Mnew[c]; DMold[c] = DMnew[c]; }
#pragma unroll
        for (int k = 0; k < RS; ++k) xc[k] = xn[k];
      }
      if constexpr (FWD_ONLY) {
        // Level k < NL of this strip: the sum of its final column sums.
#pragma unroll
        for (int k = 1; k < NL; ++k) {
          double sk = 0.0;
#pragma unroll
          for (int c = 0; c < C; ++c) sk += (double)Ccol[k - 1][c];
          lt[k] += sk;
        }
      }
      // Final column sums: read back by the adjoint pass (the last strip's
      // stay in registers when both passes run in one launch).
      if (cs_on && ((ns > 1 && s + 1 < ns) || !(phases & 2))) {
        T* dst = CS + (long long)s * NX * C * 32;
#pragma unroll
        for (int h = 0; h < NX; ++h)
#pragma unroll
          for (int c = 0; c < C; ++c) dst[(h * C + c) * 32 + lane] = Ccol[h][c];
      }
      __syncwarp();  // carries and records of this strip -> later readers
    };
    for (int s = 0; s < ((phases & 1) ? ns : 0); ++s) fwd_strip(s, !ckpt || s == ns - 1, true);
    if constexpr (FWD_ONLY) {
      // Level totals of the pair: lanes summed in a fixed order (FP64).
#pragma unroll
      for (int k = 1; k <= NL; ++k) {
        double v = lt[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        if (lane == 0 && k <= args.nl_out) args.lev[(long long)k * args.ntasks + task] = v;
      }
    }

    // ---------------- phase 2: adjoint, bottom-up, strips right to left ----
    for (int s = (phases & 2) ? ns - 1 : -1; s >= 0; --s) {
      if constexpr (CKPT) {
        if (s != ns - 1) fwd_strip(s, true, false);  // this strip's records
      }
      stage_y(s);
      if (s != ns - 1 || !(phases & 1)) {
        const T* src = CS + (long long)s * NX * C * 32;
#pragma unroll
        for (int h = 0; h < NX; ++h)
#pragma unroll
          for (int c = 0; c < C; ++c) Ccol[h][c] = src[(h * C + c) * 32 + lane];
      }
      T E[NX][C];  // adjoint column suffix sums (rows below the current row)
#pragma unroll
      for (int h = 0; h < NX; ++h)
#pragma unroll
        for (int c = 0; c < C; ++c) E[h][c] = T(0);
      T Mprev[C], argprev[C], Zbprev[C];
#pragma unroll
      for (int c = 0; c < C; ++c) { Mprev[c] = T(0); argprev[c] = T(0); Zbprev[c] = T(0); }
      T DMlast0 = T(0), mr_old = T(0), ar_old = T(0);
      T accprev[KD];
#pragma unroll
      for (int k = 0; k < KD; ++k) accprev[k] = T(0);
      T Aprev[NX];
#pragma unroll
      for (int h = 0; h < NX; ++h) Aprev[h] = T(0);
      const T* brin = BR + (long long)((s + 1) & 1) * rm * NX;  // written by strip s + 1
      T* brout = BR + (long long)(s & 1) * rm * NX;
      T xc[RS];
      load_x(lx + 31 - lane, xc);
      // Record of the row this lane processes next (prefetched one step).
      T recn[NX];
      {
        const int rho0 = -(31 - lane);
        const bool act0 = rho0 >= 1 && rho0 <= lx;
#pragma unroll
        for (int h = 0; h < NX; ++h)
          recn[h] = (act0 && NH > 0) ? rec_at(s, lx + 33)[h * 32 + lane] : T(0);
      }
      const int T2 = lx + 33;
#pragma unroll kStepUnroll2
      for (int u = 0; u < T2; ++u) {
        const int rho = u - (31 - lane);
        const int g = lx - rho;                      // grid row computed; cell row processed
        const bool act = rho >= 1 && rho <= lx;      // cell row g exists
        const bool fin = rho >= 1 && rho <= lx + 1;  // grid row g + 1 completes here
        // Values lane l+1 produced one step earlier (same rows).
        const T right = shfl_down(DMlast0, 1);
        const T mr_new = shfl_down(Mprev[0], 1);
        const T ar_new = want_dpar ? shfl_down(argprev[0], 1) : T(0);
        T Ain[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h) Ain[h] = shfl_down(Aprev[h], 1);
        T acc[KD];
#pragma unroll
        for (int k = 0; k < KD; ++k) acc[k] = shfl_down(accprev[k], 1);
        if (lane == 31) {
#pragma unroll
          for (int k = 0; k < KD; ++k) acc[k] = T(0);
#pragma unroll
          for (int h = 0; h < NX; ++h)
            Ain[h] = (s + 1 < ns && act) ? brin[(long long)g * NX + h] : T(0);
        }
        T Xin[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h) Xin[h] = recn[h];
        {
          const bool actn = rho + 1 >= 1 && rho + 1 <= lx;
          const long long tn = (long long)lx + 33 - (u + 1);
#pragma unroll
          for (int h = 0; h < NX; ++h)
            recn[h] = (actn && NH > 0) ? rec_at(s, tn)[h * 32 + lane] : T(0);
        }
        T xn[RS];
        load_x(g - 1, xn);
        T Mnew[C], argn[C];
        gram_row(xc, Mnew, argn);
        T DMnew[C];
#pragma unroll
        for (int c = 0; c < C; ++c) DMnew[c] = Mprev[c] - Mnew[c];
        T Z[C];
#pragma unroll
        for (int c = 0; c < C - 1; ++c) Z[c] = DMnew[c + 1] - DMnew[c];
        Z[C - 1] = lane == 31 ? T(0) : right - DMnew[C - 1];
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (!act || s * STRIP + C * lane + c >= ly) Z[c] = T(0);

        T Zb[C];
        T Aout[NX];
        T H[NX];
#pragma unroll
        for (int h = 0; h < NX; ++h) H[h] = Xin[h];
        if (P == 1) {
          // Q[h]: running Rbar of level h+1 (suffix over the columns right of
          // the current one); Aout: everything from this lane's first column.
          T Q[NX];
#pragma unroll
          for (int h = 0; h < NX; ++h) {
            T tsum = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c) tsum += E[h][c];
            Aout[h] = Ain[h] + tsum;
            Q[h] = w[h + 1] + Aout[h];
          }
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const T z = Z[c];
            // Forward state at (g, c): undo the row's column-sum updates.
            T cf[NX];
            T cprev = T(1);
#pragma unroll
            for (int k = 2; k <= NL; ++k) {
              Ccol[k - 2][c] = fma(-z, cprev, Ccol[k - 2][c]);
              cf[k - 2] = H[k - 2];
              H[k - 2] += Ccol[k - 2][c];
              cprev = cf[k - 2];
            }
            // Adjoint, top level down.
            T rb_next = w[NL];
            T zb;
            if constexpr (NL >= 2) zb = rb_next * cf[NL - 2];
            else zb = rb_next;
#pragma unroll
            for (int k = NL - 1; k >= 1; --k) {
              Q[k - 1] -= E[k - 1][c];
              const T rb = Q[k - 1];
              E[k - 1][c] = fma(z, rb_next, E[k - 1][c]);
              zb = (k >= 2) ? fma(rb, cf[k >= 2 ? k - 2 : 0], zb) : zb + rb;
              rb_next = rb;
            }
            Zb[c] = zb;
          }
        } else {
          // Left to right: forward state; keeps, per cell, the horizontal
          // prefixes H the cell saw (NH values).  Together with the column
          // sums (back at their values before this row) and z they give the
          // coefficient of z in every state of every level (cf below).
          T Hs[C][NX];
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const T z = Z[c];
            T Rp[P][P];
#pragma unroll
            for (int i = 0; i < P; ++i)
#pragma unroll
              for (int j = 0; j < P; ++j) Rp[i][j] = T(0);
            Rp[0][0] = z;
            T tot = z;
#pragma unroll
            for (int k = 2; k <= NL; ++k) {
              const int f = Lay::f(k), fp = Lay::f(k - 1), o = Lay::off(k);
              T Rn[P][P];
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) Rn[i][j] = T(0);
              Ccol[o][c] -= tot;
              Hs[c][o] = H[o];
              Rn[0][0] = z * H[o];
              H[o] += Ccol[o][c];
              T lsum = Rn[0][0];
#pragma unroll
              for (int rr = 1; rr < P; ++rr) {
                if (rr < f) {
                  T Vs = T(0), Us = T(0);
#pragma unroll
                  for (int i = 0; i < P; ++i)
                    if (i < fp) { Vs += Rp[i][rr - 1]; Us += Rp[rr - 1][i]; }
                  const T zr = z * (T(1) / T(rr + 1));
                  Ccol[o + rr][c] -= Vs;
                  Rn[0][rr] = zr * Ccol[o + rr][c];
                  Hs[c][o + rr] = H[o + rr];
                  Rn[rr][0] = zr * H[o + rr];
                  H[o + rr] += Us;
                  lsum += Rn[0][rr] + Rn[rr][0];
#pragma unroll
                  for (int ss = 1; ss < P; ++ss) {
                    if (ss < f) {
                      Rn[rr][ss] = z * (T(1) / T((rr + 1) * (ss + 1))) * Rp[rr - 1][ss - 1];
                      lsum += Rn[rr][ss];
                    }
                  }
                }
              }
              tot = lsum;
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) Rp[i][j] = Rn[i][j];
            }
          }
          // Coefficient of z in state (i, j) of level k at cell c:
          //   (0,0): H;  (0,j): column sum / (j+1);  (i,0): H / (i+1);
          //   (i,j): z / ((i+1)(j+1)) times the level-(k-1) coefficient of
          //   (i-1, j-1)  (ksig/algorithms.py:121-138); level 1 is 1.
          auto cf = [&](int c, int k, int i, int j) -> T {
            const T z = Z[c];
            T v = T(1);
            int kk = k, ii = i, jj = j;
#pragma unroll
            for (int t = 0; t < P; ++t) {
              if (ii >= 1 && jj >= 1) {
                v *= z * (T(1) / T((ii + 1) * (jj + 1)));
                --kk; --ii; --jj;
              }
            }
            if (kk <= 1) return v;
            const int o = Lay::off(kk);
            if (ii == 0 && jj == 0) return v * Hs[c][o];
            if (ii == 0) return v * Ccol[o + jj][c] * (T(1) / T(jj + 1));
            return v * Hs[c][o + ii] * (T(1) / T(ii + 1));
          };
          // Right to left: the adjoint, top level down.
          T Rb_next[C][P][P];
          T pendDA[P][C];
#pragma unroll
          for (int c = 0; c < C; ++c) Zb[c] = T(0);
#pragma unroll
          for (int k = NL; k >= 1; --k) {
            const int f = Lay::f(k);
            const int fn = (k < NL) ? Lay::f(k + 1) : 0;
            const int on = (k < NL) ? Lay::off(k + 1) : 0;
            T Ab = (k < NL) ? Ain[on] : T(0);
            T Ub[P];
#pragma unroll
            for (int rr = 0; rr < P; ++rr) {
              Ub[rr] = T(0);
              if (k < NL && rr >= 1 && rr < fn) Ub[rr] = Ain[on + rr];
            }
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
                      if (j + 1 < fn) v += E[on + j + 1][c];
                      if (i + 1 < fn) v += Ub[i + 1];
                      if (i + 1 < fn && j + 1 < fn)
                        v += z * (T(1) / T((i + 2) * (j + 2))) * Rb_next[c][i + 1][j + 1];
                    }
                  }
                  Rb[i][j] = v;
                }
              if (k == 1) {
                Zb[c] += Rb[0][0];
              } else {
#pragma unroll
                for (int i = 0; i < P; ++i)
#pragma unroll
                  for (int j = 0; j < P; ++j)
                    if (i < f && j < f) Zb[c] += Rb[i][j] * cf(c, k, i, j);
              }
              if (k < NL) {
                Ab += E[on][c];
#pragma unroll
                for (int rr = 1; rr < P; ++rr)
                  if (rr < fn) Ub[rr] += z * (T(1) / T(rr + 1)) * Rb_next[c][rr][0];
              }
#pragma unroll
              for (int i = 0; i < P; ++i)
#pragma unroll
                for (int j = 0; j < P; ++j) Rb_next[c][i][j] = Rb[i][j];
            }
            if (k < NL) {
              Aout[on] = Ab;
#pragma unroll
              for (int rr = 1; rr < P; ++rr)
                if (rr < fn) Aout[on + rr] = Ub[rr];
              // Level k+1's column increments go in now that level k has
              // read the suffixes of the rows below.
#pragma unroll
              for (int c = 0; c < C; ++c)
#pragma unroll
                for (int rr = 0; rr < P; ++rr)
                  if (rr < fn) E[on + rr][c] += pendDA[rr][c];
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
          if (NH == 0) Aout[0] = T(0);
        }
        // Cells outside the pair (padding, the next strip's cell) carry no
        // adjoint.
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (!act || s * STRIP + C * lane + c >= ly || (lane == 31 && c == C - 1)) Zb[c] = T(0);
        if (lane == 0 && act && s > 0) {
#pragma unroll
          for (int h = 0; h < NX; ++h) brout[(long long)g * NX + h] = Aout[h];
        }

        // ---- grid row p = g + 1: partial Mbar of this lane's cells ----
        const int p = g + 1;
        T dp = T(0), sw = T(0);
#pragma unroll
        for (int c = 0; c <= C; ++c) {
          T mb, Mq, aq;
          if (c < C) {
            mb = Zbprev[c] - Zb[c];
            if (c > 0) mb += Zb[c - 1] - Zbprev[c - 1];
            Mq = Mprev[c];
            aq = argprev[c];
          } else {
            mb = Zb[C - 1] - Zbprev[C - 1];
            Mq = mr_old;
            aq = ar_old;
          }
          const int q = s * STRIP + C * lane + c;
          const bool valid = fin && q < Ly && (c < C || lane < 31);
          const T W = valid ? (rbf ? mb * Mq : mb) : T(0);
          // RBF: column 0 is the lane's centre (y' = 0); sums in the lane's
          // frame, scaled by 2a (the stored columns are 2a y').
          if (!rbf || c > 0) {
            T yv[RS];
            y_col(c, yv);
#pragma unroll
            for (int k = 0; k < KD; ++k) acc[k] = fma(W, yv[k], acc[k]);
          }
          sw += W;
          dp = fma(W, rbf ? aq : Mq, dp);
        }
        if (want_dpar) dpar_w += (double)dp;
        if (rbf) {
          // 2a sum_c W_c (y_c - x_p) = sum_c W_c 2a y'_c - 2a x'_p sum_c W_c:
          // frame-independent, so the lanes' shares add up along the row.
          T xp[RS], negc[RS];
          load_x(p, xp);
          y_col(0, negc);
          const T t = T(-2) * ralpha * sw;
#pragma unroll
          for (int k = 0; k < KD; ++k) acc[k] = fma(xp[k] + negc[k], t, acc[k]);
        }
        if (lane == 0 && fin) {
          T* dst = args.dX + ((long long)a * args.LX + p) * args.d;
#pragma unroll
          for (int k = 0; k < KD; ++k) {
            if (k < args.d) {
              atomicAdd(dst + k, xscale_t * acc[k]);
            }
          }
        }
#pragma unroll
        for (int k = 0; k < KD; ++k) accprev[k] = acc[k];
#pragma unroll
        for (int h = 0; h < NX; ++h) Aprev[h] = Aout[h];
        DMlast0 = DMnew[0];
        mr_old = mr_new;
        ar_old = ar_new;
#pragma unroll
        for (int c = 0; c < C; ++c) { Mprev[c] = Mnew[c]; argprev[c] = argn[c]; Zbprev[c] = Zb[c]; }
#pragma unroll
        for (int k = 0; k < RS; ++k) xc[k] = xn[k];
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

template <typename T, int KD, int C, int NL, int P, int WPB>
__global__ void __launch_bounds__(WPB * 32)
dp_bwd_kernel(const DpBwdArgs<T> args) {
  if (args.kind == KIND_RBF && args.dparam == nullptr)
    dp_bwd_body<T, KD, C, NL, P, WPB, true, false>(args);
  else
    dp_bwd_body<T, KD, C, NL, P, WPB, false, false>(args);
}

// The adjoint with strip checkpointing (DpBwdArgs::ckpt): phase 1 keeps one
// strip of records, phase 2 recomputes the others from their checkpoints.
template <typename T, int KD, int C, int NL, int P, int WPB>
__global__ void __launch_bounds__(WPB * 32)
dp_bwd_ckpt_kernel(const DpBwdArgs<T> args) {
  dp_bwd_body<T, KD, C, NL, P, WPB, false, false, true>(args);
}

// Forward pass of the split gradient pass (order 1): phase 1 with per-pair
// records and level totals, in a kernel of its own so that the adjoint
// kernel's register allocation is not shared with it.
template <typename T, int KD, int C, int NL, int P, int WPB>
__global__ void __launch_bounds__(WPB * 32)
dp_rec_fwd_kernel(const DpBwdArgs<T> args) {
  static_assert(P == 1, "the split gradient pass is order 1");
  if (args.kind == KIND_RBF)
    dp_bwd_body<T, KD, C, NL, P, WPB, true, true>(args);
  else
    dp_bwd_body<T, KD, C, NL, P, WPB, false, true>(args);
}

}  // namespace ksig
