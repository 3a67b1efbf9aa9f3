// Skewed systolic sweep shared by the forward signature kernels.
//
// Work unit: one (row sequence x, column sequence y) pair.  One warp runs a
// stream of pairs.  Within a pair the cell grid (lx rows x ly columns of
// second-difference increments) is swept row by row; lane l owns C
// consecutive grid columns of a vertical strip and runs one row step behind
// lane l-1, so every left-to-right dependency of a cell row (prefix sums for
// the DP, the left K values for the PDE) arrives from lane l-1 by register
// shuffles.  Lanes continue straight into the next strip / pair, so the
// pipeline drains only once, at the end of the warp's stream.
//
// Per row step u of an item a lane:
//   1. evaluates the static kernel on grid row u+1 (or, on the last step,
//      on row 0 of its next item) for its C columns: one fused dot product
//      per grid point and an exp2 on the SFU, so the Gram never leaves
//      registers;
//   2. forms the vertical differences DM of grid rows u-1, u and, with the
//      right neighbour's first DM, the second differences Z of cell row u-1
//      (ksig/algorithms.py:63-64);
//   3. hands Z to the recursion policy (DP levels or Goursat PDE), which
//      consumes the left neighbour's exchange values and produces its own.
// Strips are 32*C-1 cells wide (the last grid column of a strip is the first
// of the next); lane 31 hands its exchange values for every row to lane 0 of
// the next strip through a per-warp boundary buffer in global scratch.
// Rows past a sequence's end and columns past its end repeat the last point,
// which makes their increments exactly zero (edge-padding invariance).
#pragma once

#include "common.cuh"

namespace ksig {

template <typename T>
struct SweepArgs {
  const T* xr;           // packed row-side points  [*, RS]
  const int64_t* xstart; // [nX] first packed row of each row sequence
  const int32_t* xlen;   // [nX] points per sequence
  const T* yr;           // packed column-side points
  const int64_t* ystart;
  const int32_t* ylen;
  int mode;              // KSIG_PAIRS_*
  int nY;                // column count for FULL decode / n for UPPER
  const int2* list;      // explicit pairs (LIST mode)
  const int* order;      // optional task permutation (longest first)
  int ntasks;
  int kind;              // static kernel
  double* out;           // per-task outputs, layout set by the policy
  T* scratch;            // boundary buffers, scratch_per_warp elements per warp
  long long scratch_per_warp;
  int multi_strip;       // some pair needs more than one strip
  int nl_out;            // levels written (<= the instantiated NL)
  int nX, nYseq;         // sequence counts (bounds of LIST pairs)
  int* status;
};

// Item geometry a policy may need.
struct ItemInfo {
  int task, Lx, Ly, s, ns;
};

template <typename T, int KD, int C, bool DIFF, int WPB, class Policy>
__device__ __forceinline__ void sweep(const SweepArgs<T>& args, Policy& pol) {
  constexpr int NX = Policy::NX;
  constexpr int RS = packed_stride<T>(KD);
  constexpr int VN = Vec<T>::N;
  using V = typename Vec<T>::type;
  constexpr int STRIP = DIFF ? 32 * C - 1 : 32 * C;

  const int lane = threadIdx.x & 31;
  const long long wg = (long long)blockIdx.x * WPB + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * WPB;
  T* bbuf = args.scratch ? args.scratch + wg * args.scratch_per_warp : nullptr;

  long long seq = 0;
  int task = -1, a = 0, b = 0, Lx = 1, Ly = 1, rows = 16, ns = 1, s = 0, u = 0;

  auto load_task = [&](long long q, int& t_, int& a_, int& b_, int& Lx_,
                       int& Ly_, int& rows_, int& ns_) {
    const long long tid = wg + q * nw;
    if (tid >= args.ntasks) {
      t_ = -1; a_ = 0; b_ = 0; Lx_ = 1; Ly_ = 1; rows_ = 16; ns_ = 1;
      return;
    }
    t_ = (int)tid;
    int2 ab = decode_task((int)tid, args.mode, args.nY, args.list, args.order);
    if (ab.x < 0 || ab.x >= args.nX || ab.y < 0 || ab.y >= args.nYseq) {
      set_status(args.status, KSIG_ERR_INVALID);  // pair index out of range
      ab = make_int2(0, 0);
    }
    a_ = ab.x; b_ = ab.y;
    Lx_ = args.xlen[a_];
    Ly_ = args.ylen[b_];
    const int lx = DIFF ? Lx_ - 1 : Lx_;
    const int ly = DIFF ? Ly_ - 1 : Ly_;
    ns_ = ly <= STRIP ? 1 : (ly + STRIP - 1) / STRIP;
    rows_ = lx > 16 ? lx : 16;
    if (ns_ > 1 && rows_ < 32) rows_ = 32;
  };

  T yv[C][KD + 1];
  const T* xbase = args.xr;
  int gLx = 1;

  auto load_y = [&](int b_, int Ly_, int s_) {
    const int g0 = s_ * STRIP + C * lane;
    const T* ybase = args.yr + args.ystart[b_] * RS;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      int col = g0 + c;
      col = col < Ly_ - 1 ? col : Ly_ - 1;
      const V* p = reinterpret_cast<const V*>(ybase + (long long)col * RS);
      T tmp[RS];
#pragma unroll
      for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(tmp)[v] = __ldg(p + v);
#pragma unroll
      for (int k = 0; k <= KD; ++k) yv[c][k] = tmp[k];
    }
  };

  auto gram_row = [&](int row, T (&m)[C]) {
    row = row < gLx - 1 ? row : gLx - 1;
    const V* p = reinterpret_cast<const V*>(xbase + (long long)row * RS);
    T xv[RS];
#pragma unroll
    for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(p + v);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      T acc = xv[KD] + yv[c][KD];
#pragma unroll
      for (int k = 0; k < KD; ++k) acc = fma(xv[k], yv[c][k], acc);
      m[c] = static_value(acc, args.kind);
    }
  };

  T Mcur[C], DMcur[C];
  load_task(0, task, a, b, Lx, Ly, rows, ns);
  xbase = args.xr + (task >= 0 ? args.xstart[a] : 0) * RS;
  gLx = Lx;
  if (task >= 0) {
    load_y(b, Ly, 0);
  } else {
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int k = 0; k <= KD; ++k) yv[c][k] = T(0);
  }
  gram_row(0, Mcur);
#pragma unroll
  for (int c = 0; c < C; ++c) DMcur[c] = T(0);
  pol.begin_item();
  if (task >= 0) pol.begin_task(ItemInfo{task, Lx, Ly, 0, ns}, lane);

  int delay = lane;
  bool done = task < 0;
  for (;;) {
    if (__all_sync(FULL, done)) break;
    const bool active = delay == 0 && !done;

    // Exchange values of the same cell row from lane l-1 (one step earlier).
    T Xin[NX];
#pragma unroll
    for (int h = 0; h < NX; ++h) Xin[h] = shfl_up(pol.X[h], 1);

    const bool last_row = (u == rows);
    int ntask = task, na = a, nb = b, nLx = Lx, nLy = Ly, nrows = rows, nns = ns, ns_next = s;
    long long nseq = seq;
    if (__any_sync(FULL, active && last_row)) {
      if (active && last_row) {
        if (s + 1 < ns) {
          ns_next = s + 1;
        } else {
          nseq = seq + 1;
          load_task(nseq, ntask, na, nb, nLx, nLy, nrows, nns);
          ns_next = 0;
        }
        if (ntask >= 0) {
          xbase = args.xr + args.xstart[na] * RS;
          gLx = nLx;
          load_y(nb, nLy, ns_next);
        }
      }
    }
    T Mnew[C];
    gram_row(last_row ? 0 : u + 1, Mnew);
    // With differencing DM holds vertical differences of grid rows; without
    // it DM carries the previous grid row (the cells of row u-1 themselves).
    T DMnew[C];
#pragma unroll
    for (int c = 0; c < C; ++c) DMnew[c] = DIFF ? Mnew[c] - Mcur[c] : Mcur[c];
    const T DMright = shfl_down(DMnew[0], 1);

    if (active && u >= 1 && task >= 0) {
      const int r = u - 1;
      if (lane == 0) {
        if (s > 0) {
          const T* src = bbuf + (long long)r * NX;
#pragma unroll
          for (int h = 0; h < NX; ++h) Xin[h] = __ldcg(src + h);
        } else {
          pol.left_boundary(Xin);
        }
      }
      T Z[C];
      if (DIFF) {
#pragma unroll
        for (int c = 0; c < C - 1; ++c) Z[c] = DMcur[c + 1] - DMcur[c];
        Z[C - 1] = DMright - DMcur[C - 1];
      } else {
        const int g0 = s * STRIP + C * lane;
#pragma unroll
        for (int c = 0; c < C; ++c)
          Z[c] = (r < Lx && g0 + c < Ly) ? DMcur[c] : T(0);
      }
      // Lane 31's last cell belongs to the next strip when differencing.
      const bool mask_last = DIFF && lane == 31;
      if (mask_last) Z[C - 1] = T(0);
      pol.row(Z, Xin, mask_last, r, ItemInfo{task, Lx, Ly, s, ns}, lane);
      if (lane == 31 && s + 1 < ns) {
        T* dst = bbuf + (long long)r * NX;
#pragma unroll
        for (int h = 0; h < NX; ++h) __stcg(dst + h, pol.X[h]);
      }
    }
    if (args.multi_strip) __syncwarp();

    bool finished_task = false;
    long long fin_seq = seq;
    int fin_task = task;
    if (active && last_row) {
      if (s + 1 >= ns && task >= 0) {
        finished_task = true;
        pol.end_task(seq, task, lane);
      }
      pol.begin_item();
      task = ntask; a = na; b = nb; Lx = nLx; Ly = nLy; rows = nrows; ns = nns;
      if (nseq != seq && task >= 0) pol.begin_task(ItemInfo{task, Lx, Ly, 0, ns}, lane);
      s = ns_next; seq = nseq; u = 0;
      if (task < 0) done = true;
    } else if (active) {
      ++u;
    }
    if (active) {
#pragma unroll
      for (int c = 0; c < C; ++c) { DMcur[c] = DMnew[c]; Mcur[c] = Mnew[c]; }
    }

    // A pair is complete once lane 31 (the last lane) has finished it.
    const int l31_fin = __shfl_sync(FULL, finished_task ? 1 : 0, 31);
    if (l31_fin) {
      const long long q = __shfl_sync(FULL, fin_seq, 31);
      const int t = __shfl_sync(FULL, fin_task, 31);
      pol.collect(q, t, lane);
    }
    if (delay > 0) --delay;
  }
}

// ---------------------------------------------------------------------------
// DP level recursion (Alg. 3 for P == 1, Alg. 6 otherwise).
// ---------------------------------------------------------------------------

template <int NL, int P>
struct DpLayout {
  __host__ __device__ static constexpr int f(int k) { return k < P ? k : P; }
  __host__ __device__ static constexpr int off(int k) {  // level k >= 2
    int o = 0;
    for (int q = 2; q < k; ++q) o += f(q);
    return o;
  }
  static constexpr int NH = off(NL + 1);
};

// Per-lane state of the level recursion.
//   order 1 (ksig/algorithms.py:78-83): R_1 = Z, R_k = Z * excl2d(R_{k-1});
//   order p (ksig/algorithms.py:121-138): R_k[0][0] = Z * excl2d(sum R_{k-1}),
//     R_k[0][r] = Z/(r+1) * excl_rows(sum_a R_{k-1}[a][r-1]),
//     R_k[r][0] = Z/(r+1) * excl_cols(sum_b R_{k-1}[r-1][b]),
//     R_k[r][s] = Z/((r+1)(s+1)) * R_{k-1}[r-1][s-1].
// The exclusive 2-D prefix at (i, j) is sum_{j'<j} colsum_{i'<i}: column
// sums live in Ccol (per lane, per column), the running sum over j' < j is
// the exchange value H handed from lane to lane.  Row prefixes (axis -1) are
// exchange values too; column prefixes (axis -2) are column sums.
template <typename T, int C, int NL, int P, int WPB>
struct DpPolicy {
  using L = DpLayout<NL, P>;
  static constexpr int NX = L::NH > 0 ? L::NH : 1;
  T X[NX];                    // horizontal running sums (outgoing)
  T Ccol[NX][C];              // column running sums
  float accs[NL + 1], accc[NL + 1];
  double accd[NL + 1];
  double (*red)[NL][32];      // this warp's [2][NL][32] reduction slots
  double* out;
  int ntasks, nl_out;

  __device__ void init(double (*red_)[NL][32], double* out_, int ntasks_, int nl_out_) {
    red = red_; out = out_; ntasks = ntasks_; nl_out = nl_out_;
#pragma unroll
    for (int k = 0; k <= NL; ++k) { accs[k] = 0.f; accc[k] = 0.f; accd[k] = 0.0; }
#pragma unroll
    for (int h = 0; h < NX; ++h) X[h] = T(0);
  }
  __device__ void begin_item() {
#pragma unroll
    for (int h = 0; h < NX; ++h)
#pragma unroll
      for (int c = 0; c < C; ++c) Ccol[h][c] = T(0);
  }
  __device__ void begin_task(const ItemInfo&, int) {}
  __device__ void left_boundary(T (&Xin)[NX]) {
#pragma unroll
    for (int h = 0; h < NX; ++h) Xin[h] = T(0);
  }

  __device__ void row(const T (&Z)[C], const T (&Xin)[NX], bool, int,
                      const ItemInfo&, int) {
    T H[NX];
#pragma unroll
    for (int h = 0; h < NX; ++h) H[h] = Xin[h];
    T rowacc[NL + 1];
#pragma unroll
    for (int k = 0; k <= NL; ++k) rowacc[k] = T(0);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const T z = Z[c];
      T Rp[P][P];
#pragma unroll
      for (int i = 0; i < P; ++i)
#pragma unroll
        for (int j = 0; j < P; ++j) Rp[i][j] = T(0);
      Rp[0][0] = z;
      rowacc[1] += z;
#pragma unroll
      for (int k = 2; k <= NL; ++k) {
        const int f = L::f(k), fp = L::f(k - 1), o = L::off(k);
        T A = T(0);
#pragma unroll
        for (int i = 0; i < P; ++i)
#pragma unroll
          for (int j = 0; j < P; ++j)
            if (i < fp && j < fp) A += Rp[i][j];
        T Rn[P][P];
#pragma unroll
        for (int i = 0; i < P; ++i)
#pragma unroll
          for (int j = 0; j < P; ++j) Rn[i][j] = T(0);
        Rn[0][0] = z * H[o];
        H[o] += Ccol[o][c];
        Ccol[o][c] += A;
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
        rowacc[k] += lsum;
#pragma unroll
        for (int i = 0; i < P; ++i)
#pragma unroll
          for (int j = 0; j < P; ++j) Rp[i][j] = Rn[i][j];
      }
    }
#pragma unroll
    for (int h = 0; h < NX; ++h) X[h] = H[h];
    // Compensated (Neumaier) accumulation of the row partials.
#pragma unroll
    for (int k = 1; k <= NL; ++k) {
      if (sizeof(T) == 8) {
        accd[k] += (double)rowacc[k];
      } else {
        const float x = (float)rowacc[k];
        const float t = accs[k] + x;
        const float e = fabsf(accs[k]) >= fabsf(x) ? (accs[k] - t) + x : (x - t) + accs[k];
        accc[k] += e;
        accs[k] = t;
      }
    }
  }

  __device__ void end_task(long long seq, int, int lane) {
#pragma unroll
    for (int k = 1; k <= NL; ++k) {
      const double v = sizeof(T) == 8 ? accd[k] : (double)accs[k] + (double)accc[k];
      red[seq & 1][k - 1][lane] = v;
      accs[k] = 0.f; accc[k] = 0.f; accd[k] = 0.0;
    }
  }

  // Warp-wide: sum the 32 lanes' level sums of task t (FP64, fixed order).
  __device__ void collect(long long q, int t, int lane) {
    __syncwarp();
#pragma unroll
    for (int k = 1; k <= NL; ++k) {
      double v = red[q & 1][k - 1][lane];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
      if (lane == 0 && k <= nl_out) out[(long long)k * ntasks + t] = v;
    }
    if (lane == 0) out[t] = 1.0;
    __syncwarp();
  }
};

template <typename T, int KD, int C, int NL, int P, bool DIFF, int WPB>
__global__ void __launch_bounds__(WPB * 32)
dp_fwd_kernel(const SweepArgs<T> args) {
  __shared__ double red[WPB][2][NL][32];
  DpPolicy<T, C, NL, P, WPB> pol;
  pol.init(red[threadIdx.x >> 5], args.out, args.ntasks, args.nl_out);
  sweep<T, KD, C, DIFF, WPB>(args, pol);
}

// ---------------------------------------------------------------------------
// Goursat PDE (ksig/algorithms.py:344-399) with dyadic refinement F = 2^k.
// ---------------------------------------------------------------------------

// Per-lane state: K at the lane's refined right edges on the current refined
// row.  The scheme of ksig/algorithms.py:384-385 (q = Z / F^2 per refined cell)
//   K[i+1,j+1] = (K[i,j+1] + K[i+1,j]) (1 + q/2 + q^2/12) - K[i,j] (1 - q^2/12)
// is evaluated in increment form: with H = K[i+1,j+1] - K[i,j+1] (the vertical
// increment, accumulated along the row) and
//   g = (K[i,j+1] + K[i+1,j]) (q/2 + q^2/12) + K[i,j] q^2/12,
// H[j+1] = H[j] + g and K[i+1,j+1] = K[i,j+1] + H[j+1].  This is the same
// recurrence, but FP32 rounding errors then grow with i + j instead of i * j
// (the plain form loses ~3e-4 relative on 600 x 500 refined grids; this form
// stays near 1e-6).  Exchange values per refined row: K and H at the lane's
// right boundary.
template <typename T, int C, int F, bool DIFF>
struct PdePolicy {
  static constexpr int NX = 2 * F;
  static constexpr int STRIP = DIFF ? 32 * C - 1 : 32 * C;
  T X[NX];
  T Kr[C * F];
  T kcorner;     // K at the lane's left boundary on the row above the block
  double* out;
  int tgt_s, tgt_lane, tgt_c, tgt_r;  // where the far corner of the pair lives

  __device__ void init(double* out_) {
    out = out_;
    tgt_s = -1; tgt_lane = -1; tgt_c = 0; tgt_r = -1;
#pragma unroll
    for (int f = 0; f < F; ++f) { X[f] = T(1); X[F + f] = T(0); }
  }
  __device__ void begin_item() {
#pragma unroll
    for (int j = 0; j < C * F; ++j) Kr[j] = T(1);
    kcorner = T(1);
  }
  // Locates the far corner (last cell row, last cell column) of the pair.
  __device__ void begin_task(const ItemInfo& it, int lane) {
    const int lx = DIFF ? it.Lx - 1 : it.Lx;
    const int ly = DIFF ? it.Ly - 1 : it.Ly;
    if (lx <= 0 || ly <= 0) {
      tgt_s = -1; tgt_r = -1;
      if (lane == 0) out[it.task] = 1.0;  // no cells: boundary value
      return;
    }
    tgt_r = lx - 1;
    const int col = ly - 1;
    tgt_s = col / STRIP;
    const int rem = col - tgt_s * STRIP;
    tgt_lane = rem / C;
    tgt_c = rem - tgt_lane * C;
  }
  __device__ void left_boundary(T (&Xin)[NX]) {
#pragma unroll
    for (int f = 0; f < F; ++f) { Xin[f] = T(1); Xin[F + f] = T(0); }
  }

  __device__ void row(const T (&Z)[C], const T (&Xin)[NX], bool mask_last, int r,
                      const ItemInfo& it, int lane) {
    T a[C], b[C];
    constexpr T inv = T(1) / T(F * F);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const T q = Z[c] * inv;
      b[c] = q * q * (T(1) / T(12));
      a[c] = fma(T(0.5), q, b[c]);
    }
#pragma unroll
    for (int f = 0; f < F; ++f) {
      T klo = (f == 0) ? kcorner : Xin[f > 0 ? f - 1 : 0];
      T kln = Xin[f];
      T H = Xin[F + f];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const bool skip = (c == C - 1) && mask_last;
#pragma unroll
        for (int g = 0; g < F; ++g) {
          const int J = c * F + g;
          const T kro = Kr[J];
          const T gg = fma(kro + kln, a[c], klo * b[c]);
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
    kcorner = Xin[F - 1];
    if (r == tgt_r && it.s == tgt_s && lane == tgt_lane) {
      // Arithmetic select keeps Kr in registers (no dynamic indexing).
      T captured = T(0);
#pragma unroll
      for (int c = 0; c < C; ++c)
        captured = fma(T(c == tgt_c ? 1 : 0), Kr[c * F + F - 1], captured);
      out[it.task] = (double)captured;
    }
  }
  __device__ void end_task(long long, int, int) {}
  __device__ void collect(long long, int, int) {}
};

template <typename T, int KD, int C, int F, bool DIFF, int WPB>
__global__ void __launch_bounds__(WPB * 32)
pde_fwd_kernel(const SweepArgs<T> args) {
  PdePolicy<T, C, F, DIFF> pol;
  pol.init(args.out);
  sweep<T, KD, C, DIFF, WPB>(args, pol);
}

}  // namespace ksig
