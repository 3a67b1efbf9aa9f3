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

#include <cuda_pipeline.h>

#include <type_traits>

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
  StaticParams sp;       // epilogue constants of the other static kernels (EXT)
  T ralpha;              // RBF: log2(e) / max(2 s^2, 1e-12) (lane-centred Gram)
  // Gram-input instantiations (KD == 0): static-kernel values precomputed
  // by gram_kernel (gram.cuh), one [rows][gram_ld] slot per task of this
  // launch; the launch covers task positions task_base .. task_base +
  // ntasks - 1 of a call with ntasks_total tasks.
  const T* gram;
  long long gram_slot;   // elements per slot
  int gram_ld;           // row stride of a slot
  int task_base, ntasks_total;
  // Gram input: every lane reads a new slot row each step; with
  // x_prefetch > 0 it prefetches (L2) the row x_prefetch steps ahead.
  int x_prefetch;
  // Visiting order.  0: warp w takes task positions w, w + W, w + 2W, ...
  // (W warps in the grid).  > 0 (FULL or UPPER pairs, no task
  // permutation): warp w takes the visit_per consecutive entries
  // w * visit_per, ... of the column-major pair order (column b: rows
  // 0 .. nX-1, or 0 .. b of the upper triangle), so consecutive pairs of a
  // warp share their column sequence and the lanes keep their column
  // points across the switch.
  long long visit_per;
  // > 0 (with visit_per, DP policies, differencing, one strip per pair, row
  // sequences of stack_len >= 17 points each): the pairs of one column in a
  // warp's block run as one item of stacked row sequences.  The cell row
  // between two stacked sequences gets Z = 0, and each lane folds the level
  // totals of the pair above it and clears its state there (fold_pair), so
  // the pairs in between need no item switch.
  int stack_len;
};

// Item geometry a policy may need.
struct ItemInfo {
  int task, Lx, Ly, s, ns;
};

// Smem slot per lane for the next item's column points (cp.async staging);
// the kernels take WPB of these as dynamic shared memory
// (sweep_dyn_smem_bytes on the host).
template <typename T, int KD, int C>
struct SweepSmem {
  static constexpr int RS = KD == 0 ? 1 : packed_stride<T>(KD);
  T ynext[32][C * RS];
};

// Per-warp ring of item descriptors.  Every lane of a warp visits the same
// items in the same order, lane 0 first (the other lanes follow 1..31 steps
// behind), so lane 0 decodes each new pair once and leaves its geometry
// here; the other lanes copy it when they reach that pair.  Items span at
// least 16 row steps, so lane 31 trails lane 0 by at most 2 items, well
// inside the ring.
template <typename T>
struct ItemMeta {
  const T* xb;
  int task, b, Lx, Ly, rows, ns;
};
constexpr int kItemRing = 8;

template <typename T, int KD, int C, bool DIFF, int WPB, bool EXT, class Policy>
__device__ __forceinline__ void sweep(const SweepArgs<T>& args, Policy& pol,
                                      SweepSmem<T, KD, C>& sm, ItemMeta<T>* ring) {
  constexpr int NX = Policy::NX;
  // KD == 0: Gram input.  The per-step "x row" of a lane is then its C
  // static-kernel values of that grid row, read from the task's Gram slot.
  constexpr bool GIN = KD == 0;
  constexpr int RS = GIN ? C : packed_stride<T>(KD);
  constexpr int VN = Vec<T>::N;
  using V = typename Vec<T>::type;
  constexpr int STRIP = DIFF ? 32 * C - 1 : 32 * C;
  constexpr bool kPairArg = Policy::kPairArg && KD <= 16;
  // Stacking needs a few registers per lane (nb, nf, pbnd): only tiles of
  // up to 12 coordinates, where they fit without spilling (d = 32, 2
  // columns, m = 10 went from 0 to 210 bytes of spills with them).
  constexpr bool kStackable = DIFF && !GIN && Policy::kStack && KD <= 12;
  const bool stack_on = kStackable && args.stack_len > 0 && args.visit_per > 0;
  if constexpr (kStackable) pol.set_stack(stack_on ? args.stack_len : 0, args.nY);

  const int lane = threadIdx.x & 31;
  const long long wg = (long long)blockIdx.x * WPB + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * WPB;
  T* bbuf = args.scratch ? args.scratch + wg * args.scratch_per_warp : nullptr;
  T* yslot = sm.ynext[lane];

  // One item = one strip of one pair, or Lx / stack_len stacked pairs of
  // one column (task is then the first pair's, the others follow nY apart).
  struct Item {
    const T* xb;  // first packed row of the row sequence
    long long seq;
    int task, b, Lx, Ly, rows, ns, s;
  };
  // Upper triangle of K(X) in column-major order: column b holds rows
  // 0 .. b, from position b (b + 1) / 2 on.  tri_col inverts that; the
  // output slot of pair (a, b) is its row-major position upper_task.
  const bool upper = args.mode == KSIG_PAIRS_UPPER;
  auto tri_col = [&](long long p) {
    long long b = (long long)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    if (b < 0) b = 0;
    while (b > 0 && b * (b + 1) / 2 > p) --b;
    while ((b + 1) * (b + 2) / 2 <= p) ++b;
    return b;
  };
  auto upper_task = [&](long long a, long long b) {
    return (int)(a * args.nY - a * (a - 1) / 2 + (b - a));
  };

  auto make_item = [&](long long q, Item& it) {
    it.seq = q;
    it.s = 0;
    int np = 1;  // stacked pairs
    long long tid;
    int2 ab;
    if (stack_on) {
      // Run q of this warp's block: the pairs of its q-th column.
      const long long p0 = wg * args.visit_per;
      long long pend = p0 + args.visit_per;
      if (pend > args.ntasks) pend = args.ntasks;
      const long long b0 = p0 / args.nX;
      const long long start = q == 0 ? p0 : (b0 + q) * args.nX;
      long long end = (b0 + q + 1) * args.nX;
      if (end > pend) end = pend;
      tid = start < end ? start : args.ntasks;
      if (tid < args.ntasks) {
        const int b = (int)(start / args.nX);
        ab = make_int2((int)(start - (long long)b * args.nX), b);
        it.task = ab.x * args.nY + ab.y;
        np = (int)(end - start);
      }
    } else if (!GIN && args.visit_per > 0 && !upper) {
      // Column-major block of this warp (FULL pairs, natural task order).
      const long long p = wg * args.visit_per + q;
      tid = (q < args.visit_per && p < args.ntasks) ? p : args.ntasks;
      if (tid < args.ntasks) {  // p < ntasks fits an int
        const int pi = (int)p;
        const int b = pi / args.nX;
        ab = make_int2(pi - b * args.nX, b);
        it.task = ab.x * args.nY + ab.y;
      }
    } else if (!GIN && args.visit_per > 0) {
      // Upper triangle: the q-th pair of this warp's column-major block
      // (column b: rows 0 .. b).
      const long long p0 = wg * args.visit_per;
      long long pend = p0 + args.visit_per;
      if (pend > args.ntasks) pend = args.ntasks;
      const long long start = p0 + q;
      tid = start < pend ? start : args.ntasks;
      if (tid < args.ntasks) {
        const long long b = tri_col(start);
        const long long a = start - b * (b + 1) / 2;
        ab = make_int2((int)a, (int)b);
        it.task = upper_task(a, b);
      }
    } else {
      tid = wg + q * nw;
      if (tid < args.ntasks) {
        const int pos = args.task_base + (int)tid;
        it.task = args.order ? args.order[pos] : pos;
        ab = decode_task(pos, args.mode, args.nY, args.list, args.order);
      }
    }
    if (tid >= args.ntasks) {
      it.task = -1; it.b = 0; it.Lx = 1; it.Ly = 1; it.rows = 16; it.ns = 1;
      it.xb = GIN ? args.gram : args.xr;
      return;
    }
    if (ab.x < 0 || ab.x >= args.nX || ab.y < 0 || ab.y >= args.nYseq) {
      set_status(args.status, KSIG_ERR_INVALID);  // pair index out of range
      ab = make_int2(0, 0);
    }
    it.b = ab.y;
    it.xb = GIN ? args.gram + tid * args.gram_slot : args.xr + args.xstart[ab.x] * RS;
    it.Lx = np > 1 ? np * args.stack_len : args.xlen[ab.x];
    it.Ly = args.ylen[ab.y];
    const int lx = DIFF ? it.Lx - 1 : it.Lx;
    const int ly = DIFF ? it.Ly - 1 : it.Ly;
    it.ns = ly <= STRIP ? 1 : (ly + STRIP - 1) / STRIP;
    it.rows = lx > 16 ? lx : 16;
    if (it.ns > 1 && it.rows < 32) it.rows = 32;
  };
  // from_ring: called in a lane's own item switch (divergent), where lane 0
  // decodes the pair and the others copy its descriptor (ItemMeta).
  auto next_of = [&](const Item& cur, Item& nx, bool from_ring) {
    if (cur.task >= 0 && cur.s + 1 < cur.ns) {
      nx = cur;
      nx.s = cur.s + 1;
      return;
    }
    const long long q = cur.seq + 1;
    if (!from_ring) {
      make_item(q, nx);
      return;
    }
    ItemMeta<T>& m = ring[q & (kItemRing - 1)];
    if (lane == 0) {
      make_item(q, nx);
      m.xb = nx.xb; m.task = nx.task; m.b = nx.b; m.Lx = nx.Lx; m.Ly = nx.Ly;
      m.rows = nx.rows; m.ns = nx.ns;
    } else {
      nx.seq = q; nx.s = 0;
      nx.xb = m.xb; nx.task = m.task; nx.b = m.b; nx.Lx = m.Lx; nx.Ly = m.Ly;
      nx.rows = m.rows; nx.ns = m.ns;
    }
  };
  auto ycol_ptr = [&](const Item& it, int c) {
    int col = it.s * STRIP + C * lane + c;
    col = col < it.Ly - 1 ? col : it.Ly - 1;
    return args.yr + (args.ystart[it.b] + col) * RS;
  };
  // Two items with the same column sequence and strip give every lane the
  // same column points (the column-major visiting order makes this the
  // common case): the switch between them keeps the lane's registers.
  auto same_y = [&](const Item& p, const Item& n) {
    return !GIN && p.task >= 0 && n.task >= 0 && p.b == n.b && p.s == n.s;
  };
  // Stages the lane's column points of `it` into its smem slot.
  auto stage_y = [&](const Item& it) {
    if (GIN || it.task < 0) return;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const T* src = ycol_ptr(it, c);
#pragma unroll
      for (int v = 0; v < RS / VN; ++v)
        __pipeline_memcpy_async(yslot + c * RS + v * VN, src + v * VN, 16);
    }
    __pipeline_commit();
  };

  T yv[C][KD + 1];
  // RBF: the lane's columns in its centred frame (rbf_center_cols).
  const bool centred = !EXT && args.kind == KIND_RBF;
  auto y_from_slot = [&]() {
    if constexpr (GIN) return;
    __pipeline_wait_prior(0);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      T tmp[RS];
#pragma unroll
      for (int v = 0; v < RS / VN; ++v)
        reinterpret_cast<V*>(tmp)[v] = reinterpret_cast<const V*>(yslot + c * RS)[v];
#pragma unroll
      for (int k = 0; k <= KD; ++k) yv[c][k] = tmp[k];
    }
    if (centred) rbf_center_cols<KD, C>(yv, args.ralpha);
  };
  auto load_x = [&](const Item& it, int row, T (&xv)[RS]) {
    row = row < it.Lx - 1 ? row : it.Lx - 1;
    if constexpr (GIN) {
      // The lane's C Gram values of grid row `row` (columns past the
      // sequence's end repeat its last column, as the points do).
      const T* p = it.xb + (long long)row * args.gram_ld;
      const int c0 = it.s * STRIP + C * lane;
#pragma unroll
      for (int c = 0; c < C; ++c) xv[c] = __ldg(p + (c0 + c < it.Ly - 1 ? c0 + c : it.Ly - 1));
      // Every lane reads fresh slot memory each step (its own columns of a
      // new row): prefetch the row x_prefetch steps ahead into L2.
      if (args.x_prefetch > 0) {
        const int pr = row + args.x_prefetch < it.Lx - 1 ? row + args.x_prefetch : it.Lx - 1;
        const int pc = c0 < it.Ly - 1 ? c0 : it.Ly - 1;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(it.xb + (long long)pr * args.gram_ld + pc));
      }
    } else {
      const V* p = reinterpret_cast<const V*>(it.xb + (long long)row * RS);
#pragma unroll
      for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(xv)[v] = __ldg(p + v);
    }
  };
  // Static-kernel values of one grid row; call sites pass a literal for RBF,
  // so after inlining the steady loop carries no per-point select.  RBF
  // rows are moved to the lane's centred frame first; column 0 is the
  // centre itself (arg = -a |x'|^2, no dot product).
  auto gram = [&](bool RBF, const T (&xv)[RS], T (&m)[C]) {
    if constexpr (GIN) {
#pragma unroll
      for (int c = 0; c < C; ++c) m[c] = xv[c];
    } else {
      if (RBF) {
        T xt[RS];
        rbf_center_row<KD>(xv, yv[0], args.ralpha, xt);
        m[0] = kexp2(xt[KD]);
#pragma unroll
        for (int c = 1; c < C; ++c) m[c] = kexp2(centred_arg<KD, kPairArg>(xt, yv[c], xt[KD]));
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) m[c] = packed_arg<KD, kPairArg>(xv, yv[c], T(0));
      }
    }
  };
  // Runtime-kind version for the rare paths (one copy of the code).  The
  // EXT instantiations serve the other static kernels: the squared
  // distance is summed from coordinate differences (row points are packed
  // as 2x, so x is exact), which keeps it accurate for nearby points where
  // |x|^2 + |y|^2 - 2<x,y> would cancel (the Matern kernels have a cusp
  // there).
  auto gram_rt = [&](const T (&xv)[RS], T (&m)[C]) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      if constexpr (EXT) {
        T acc = T(0);
        if (args.kind == KIND_POLY) {
#pragma unroll
          for (int k = 0; k < KD; ++k) acc = fma(xv[k], yv[c][k], acc);
        } else {
#pragma unroll
          for (int k = 0; k < KD; ++k) {
            const T dk = fma(T(0.5), xv[k], -yv[c][k]);
            acc = fma(-dk, dk, acc);
          }
        }
        m[c] = static_value_other(acc, args.kind, args.sp);
      }
    }
    if constexpr (!EXT) gram(centred, xv, m);
  };

  Item cur, nxt;
  make_item(0, cur);
  next_of(cur, nxt, false);
  // First item's columns straight into registers; the next item is staged.
  if (!GIN && cur.task >= 0) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const V* p = reinterpret_cast<const V*>(ycol_ptr(cur, c));
      T tmp[RS];
#pragma unroll
      for (int v = 0; v < RS / VN; ++v) reinterpret_cast<V*>(tmp)[v] = __ldg(p + v);
#pragma unroll
      for (int k = 0; k <= KD; ++k) yv[c][k] = tmp[k];
    }
    if (centred) rbf_center_cols<KD, C>(yv, args.ralpha);
  } else {
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int k = 0; k <= KD; ++k) yv[c][k] = T(0);
  }
  if (!same_y(cur, nxt)) stage_y(nxt);

  const bool rbf = args.kind == KIND_RBF;
  // Gram input serves every static kind through the steady loop.
  const bool fast = GIN || (!EXT && (rbf || args.kind == KIND_LINEAR));
  T Mcur[C], DMcur[C], Mtmp[C], DMtmp[C];
  T xv[RS];
  load_x(cur, 0, xv);
  gram_rt(xv, Mcur);
#pragma unroll
  for (int c = 0; c < C; ++c) DMcur[c] = T(0);
  load_x(cur, 1, xv);  // Gram row of the first step

  // Cell work recorded at one step and executed at the next, so that a
  // step's Gram and its cell recursion form one branch-free block the
  // compiler can interleave.  The record holds the cells' Z directly.
  // `pit` is the item of the recorded row.
  bool pv = false, plast = false;
  int pr = 0;
  Item pit = cur;
  T pZ[C];
#pragma unroll
  for (int c = 0; c < C; ++c) pZ[c] = T(0);

  int u = 0;
  int delay = lane;
  bool done = cur.task < 0;
  // Stacked pairs: nb is the step position whose recorded row is the next
  // separator of cur; nf counts this lane's finished pairs (the reduction
  // slot parity, the same sequence in every lane).  The pair of a recorded
  // row r of a stacked item is (r + 1) / stack_len.
  constexpr int kNoBound = 0x7fffffff;
  int nb = (stack_on && cur.Lx > args.stack_len) ? args.stack_len : kNoBound;
  bool pbnd = false;
  unsigned nf = 0;

  // Cells of the recorded row + Gram of the next grid row (into Mn, with
  // vertical differences DMn against Mc).  `pvf` is false only when nothing
  // was recorded (pZ is zero then).
  auto main_block = [&](int rbf_c, bool pvf, const T (&Mc)[C], T (&Mn)[C], T (&DMn)[C],
                        T& DMright) {
    if constexpr (kStackable) {
      // The recorded row separates two stacked pairs (its Z is zero); the
      // state holds the upper pair's final column sums: fold them and
      // clear the state.  A stacked pair is complete once lane 31 has
      // folded it.  Both branches come first in the step, ahead of the
      // Gram and the recursion, which stay one block for the scheduler.
      if (pbnd) {
        pol.fold_pair(nf, lane);
        ++nf;
      }
      if (Policy::kCollect && stack_on && __shfl_sync(FULL, pbnd ? 1 : 0, 31)) {
        const long long q = (long long)__shfl_sync(FULL, nf, 31) - 1;
        const int t = __shfl_sync(FULL, pit.task + ((pr + 1) / args.stack_len - 1) * args.nY, 31);
        pol.collect(q, t, lane);
      }
    }
    T Xin[NX];
#pragma unroll
    for (int h = 0; h < NX; ++h) Xin[h] = shfl_up(pol.X[h], 1);
    if (lane == 0) {
      if (pit.s > 0 && pvf) {
        const T* src = bbuf + (long long)pr * NX;
#pragma unroll
        for (int h = 0; h < NX; ++h) Xin[h] = __ldcg(src + h);
      } else {
        pol.left_boundary(Xin);
      }
    }
    // Lane 31's last cell belongs to the next strip when differencing.
    const bool mask_last = DIFF && lane == 31;
    pol.row(pZ, Xin, mask_last, pvf, pr, ItemInfo{pit.task, pit.Lx, pit.Ly, pit.s, pit.ns}, lane);
    if (lane == 31 && pvf && pit.s + 1 < pit.ns) {
      T* dst = bbuf + (long long)pr * NX;
#pragma unroll
      for (int h = 0; h < NX; ++h) __stcg(dst + h, pol.X[h]);
    }
    if (rbf_c < 0) gram_rt(xv, Mn);  // -1: kind decided at run time
    else gram(rbf_c != 0, xv, Mn);
    // With differencing DM holds vertical differences of grid rows; without
    // it DM carries the previous grid row (the cells of row u-1 themselves).
#pragma unroll
    for (int c = 0; c < C; ++c) DMn[c] = DIFF ? Mn[c] - Mc[c] : Mc[c];
    DMright = shfl_down(DMn[0], 1);
    if (args.multi_strip) __syncwarp();
  };
  // Z of cell row u-1 of `cur` from its vertical differences DMc.
  auto record = [&](const T (&DMc)[C], T DMright, bool rec) {
    if (DIFF) {
#pragma unroll
      for (int c = 0; c < C - 1; ++c) pZ[c] = rec ? DMc[c + 1] - DMc[c] : T(0);
      pZ[C - 1] = (rec && lane != 31) ? DMright - DMc[C - 1] : T(0);
      if constexpr (kStackable) {
        // Cell row u-1 lies between two stacked sequences (grid rows
        // j*stack_len - 1 and j*stack_len): no cell, Z = 0.
        pbnd = rec && u == nb;
        if (pbnd) {
          nb += args.stack_len;
#pragma unroll
          for (int c = 0; c < C; ++c) pZ[c] = T(0);
        }
      }
    } else {
      const int g0 = cur.s * STRIP + C * lane;
#pragma unroll
      for (int c = 0; c < C; ++c)
        pZ[c] = (rec && u - 1 < cur.Lx && g0 + c < cur.Ly) ? DMc[c] : T(0);
    }
  };
  // Gram x row of the position two steps ahead (after u+1), for the
  // two-deep x prefetch of the unrolled steady loop.
  auto load_x2 = [&](T (&dst)[RS]) {
    const int u1 = u + 1;
    if (u1 < cur.rows) load_x(cur, u1 + 1, dst);
    else if (u1 == cur.rows) load_x(nxt, 0, dst);
    else load_x(nxt, 1, dst);
  };
  // One step of the steady loop (see below).
  auto steady_step = [&](int rbf_c, T (&Mc)[C], T (&Mn)[C], T (&DMc)[C], T (&DMn)[C]) {
    T DMright;
    main_block(rbf_c, true, Mc, Mn, DMn, DMright);
    record(DMc, DMright, true);
    pr = u - 1;
    ++u;
    const bool sw = (u == cur.rows);
    load_x(sw ? nxt : cur, sw ? 0 : u + 1, xv);
  };
  // Same, with this step's x row in xa, refilled afterwards with the row two
  // steps ahead (hides the strided row loads behind a whole step).
  auto steady_step2 = [&](int rbf_c, T (&Mc)[C], T (&Mn)[C], T (&DMc)[C], T (&DMn)[C],
                          T (&xa)[RS]) {
#pragma unroll
    for (int k = 0; k < RS; ++k) xv[k] = xa[k];
    T DMright;
    main_block(rbf_c, true, Mc, Mn, DMn, DMright);
    record(DMc, DMright, true);
    pr = u - 1;
    ++u;
    load_x2(xa);
  };
  auto steady_run = [&](int rbf_c, int n) {
    int it = 0;
    if (Policy::kUnroll2) {
      if (n >= 2) {
        // xa: this step's row (in xv now); xb2: the next step's row.
        T xa[RS], xb2[RS];
#pragma unroll
        for (int k = 0; k < RS; ++k) xa[k] = xv[k];
        {
          const bool sw = (u + 1 == cur.rows);
          load_x(sw ? nxt : cur, sw ? 0 : u + 2, xb2);
        }
        for (; it + 1 < n; it += 2) {  // unrolled by two: buffers swap roles
          steady_step2(rbf_c, Mcur, Mtmp, DMcur, DMtmp, xa);
          steady_step2(rbf_c, Mtmp, Mcur, DMtmp, DMcur, xb2);
        }
#pragma unroll
        for (int k = 0; k < RS; ++k) xv[k] = xa[k];  // the next step's row
      }
    } else {
      for (; it + 1 < n; ++it) {
        steady_step(rbf_c, Mcur, Mtmp, DMcur, DMtmp);
#pragma unroll
        for (int c = 0; c < C; ++c) { Mcur[c] = Mtmp[c]; DMcur[c] = DMtmp[c]; }
      }
    }
    if (it < n) {
      steady_step(rbf_c, Mcur, Mtmp, DMcur, DMtmp);
#pragma unroll
      for (int c = 0; c < C; ++c) { Mcur[c] = Mtmp[c]; DMcur[c] = DMtmp[c]; }
    }
  };

  for (;;) {
    if (__all_sync(FULL, done && !pv)) break;

    // ---- steady run: steps without any item event in any lane ----------
    // A step is plain for a lane when it is active, its recorded row is not
    // the first of an item (pr >= 1, i.e. u >= 3) and it is not the item's
    // last step (u < rows); then no item switch, no begin/end hook and no
    // pair completion happens, and every lane has a recorded row.
    {
      // (RBF and linear only: the other static kernels take the general
      // step with the run-time epilogue.)
      const bool plain = fast && delay == 0 && !done && u >= 3 && u < cur.rows;
      const int nplain = __reduce_min_sync(FULL, plain ? cur.rows - u : 0);
      if (nplain > 0) {
        if (rbf) steady_run(1, nplain);
        else steady_run(0, nplain);
        continue;
      }
    }

    // ---- general step ----------------------------------------------------
    const bool active = delay == 0 && !done;
    const bool last_row = (u == cur.rows);

    // Rare, uniform branches: item switches.
    if (__any_sync(FULL, active && last_row)) {
      if (active && last_row && nxt.task >= 0 && !same_y(cur, nxt)) y_from_slot();
    }
    if (__any_sync(FULL, pv && pr == 0)) {
      if (pv && pr == 0) {
        pol.begin_item();
        if (pit.s == 0) pol.begin_task(ItemInfo{pit.task, pit.Lx, pit.Ly, pit.s, pit.ns}, lane);
      }
    }

#pragma unroll
    for (int c = 0; c < C; ++c) pZ[c] = pv ? pZ[c] : T(0);
    T DMright;
    main_block(-1, pv, Mcur, Mtmp, DMtmp, DMright);

    // End of a recorded item / pair (rare, uniform).
    const bool fin_item = pv && plast;
    bool fin = false;
    if (__any_sync(FULL, fin_item)) {
      if (fin_item) {
        pol.end_item();
        if (pit.s + 1 >= pit.ns) {
          pol.end_task(kStackable ? (long long)nf : pit.seq, pit.task, lane);
          fin = true;
        }
      }
      // A pair is complete once lane 31 (the last lane) has finished it (of
      // a stacked item, the last pair, (pr + 1) / stack_len).
      if (__shfl_sync(FULL, fin ? 1 : 0, 31)) {
        const long long q = kStackable ? (long long)__shfl_sync(FULL, nf, 31)
                                       : __shfl_sync(FULL, pit.seq, 31);
        const int last = stack_on ? (pr + 1) / args.stack_len : 0;
        const int t = __shfl_sync(FULL, pit.task + last * args.nY, 31);
        pol.collect(q, t, lane);
      }
      if (kStackable && fin) ++nf;
    }

    // Record cell row u-1 for the next step, advance.
    const bool rec = active && u >= 1 && cur.task >= 0;
    record(DMcur, DMright, rec);
    pr = rec ? u - 1 : pr;
    plast = rec && last_row;
    pv = rec;
    if (active) {
#pragma unroll
      for (int c = 0; c < C; ++c) { DMcur[c] = DMtmp[c]; Mcur[c] = Mtmp[c]; }
      ++u;
    }
    // Item switch of the position (rare, uniform).
    if (__any_sync(FULL, (active && last_row) || (rec && u == 2))) {
      // pit: the item of the recorded rows, from cur's first recorded row
      // on (it still names cur when cur's last row runs, after the switch).
      if (rec && u == 2) pit = cur;
      if (active && last_row) {
        cur = nxt;
        next_of(cur, nxt, true);
        if (cur.task < 0) done = true;
        else if (!same_y(cur, nxt)) stage_y(nxt);
        u = 0;
        nb = (stack_on && cur.Lx > args.stack_len) ? args.stack_len : kNoBound;
      }
      // Orders lane 0's ring entry (next_of) before the other lanes read it
      // at their own switches, one or more steps later.
      __syncwarp();
    }
    // Prefetch the x row of the next step's Gram.
    {
      const bool sw = (u == cur.rows);
      load_x(sw ? nxt : cur, sw ? 0 : u + 1, xv);
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
// Level totals need no extra work per cell: the column sum of sum R_k is
// already kept for level k+1, so level k = sum_j Ccol at the end of a strip
// (one more column sum for the last level).  Strip totals are reduced in
// FP64.
template <typename T, int C, int NL, int P, int WPB>
struct DpPolicy {
  using L = DpLayout<NL, P>;
  static constexpr int NX = L::NH > 0 ? L::NH : 1;
  // Two-step unrolling of the steady loop only while the register state is
  // small enough not to spill.
  static constexpr bool kUnroll2 = P == 1 && (NX + 3) * C <= 40 && sizeof(T) == 4;
  // Paired FP32 Gram arguments (packed_arg): the wide strips of the deeper
  // truncations and the 4-column higher-order tiles, where the register
  // count and occupancy stay the same.
  static constexpr bool kPairArg = sizeof(T) == 4 && NL >= 5 && (C >= 7 || (P >= 2 && C >= 4));
  // Stacked pairs (SweepArgs::stack_len) end with fold_pair.  Order 1
  // only: the order-p state leaves no registers for the stacking counters
  // (d = 16, 4 columns, m = 8, p = 2 spilled 116 bytes with them).
  static constexpr bool kStack = P == 1;
  // Stacked pairs end in a warp-wide reduction of their level totals.
  static constexpr bool kCollect = true;
  __device__ void set_stack(int, int) {}
  T X[NX];                    // horizontal running sums (outgoing)
  T Ccol[NX][C];              // column running sums
  T Clast[C];                 // column sums of the last level's totals
  double accd[NL + 1];        // per-lane level totals of finished strips
  double (*red)[NL][32];      // this warp's [2][NL][32] reduction slots
  double* out;
  int ntasks, nl_out;

  __device__ void init(double (*red_)[NL][32], double* out_, int ntasks_, int nl_out_) {
    red = red_; out = out_; ntasks = ntasks_; nl_out = nl_out_;
#pragma unroll
    for (int k = 0; k <= NL; ++k) accd[k] = 0.0;
#pragma unroll
    for (int h = 0; h < NX; ++h) X[h] = T(0);
  }
  __device__ void begin_item() {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      Clast[c] = T(0);
#pragma unroll
      for (int h = 0; h < NX; ++h) Ccol[h][c] = T(0);
    }
  }
  __device__ void begin_task(const ItemInfo&, int) {}
  __device__ void left_boundary(T (&Xin)[NX]) {
#pragma unroll
    for (int h = 0; h < NX; ++h) Xin[h] = T(0);
  }

  // Branch-free; with all Z = 0 (no recorded row) the state is unchanged
  // apart from X, which no active neighbour reads then.
  __device__ void row(const T (&Z)[C], const T (&Xin)[NX], bool, bool, int,
                      const ItemInfo&, int) {
    if constexpr (P == 1) {
      row_order1(Z, Xin);
    } else {
      row_order_p(Z, Xin);
    }
  }

  // Order p >= 2 (Alg. 6).
  __device__ void row_order_p(const T (&Z)[C], const T (&Xin)[NX]) {
    T H[NX];
#pragma unroll
    for (int h = 0; h < NX; ++h) H[h] = Xin[h];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const T z = Z[c];
      T Rp[P][P];
#pragma unroll
      for (int i = 0; i < P; ++i)
#pragma unroll
        for (int j = 0; j < P; ++j) Rp[i][j] = T(0);
      Rp[0][0] = z;
      T tot = z;  // sum of the current level's states
#pragma unroll
      for (int k = 2; k <= NL; ++k) {
        const int f = L::f(k), fp = L::f(k - 1), o = L::off(k);
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
      Clast[c] += tot;
    }
#pragma unroll
    for (int h = 0; h < NX; ++h) X[h] = H[h];
  }

  // Order 1: R_k = z * H_k is never materialised; the column sum of level k
  // takes it straight in (Ccol_{k+1} += z * H_k, one FFMA), so a level costs
  // one FADD (the horizontal prefix) and one FFMA per cell.
  __device__ void row_order1(const T (&Z)[C], const T (&Xin)[NX]) {
    T H[NX];
#pragma unroll
    for (int h = 0; h < NX; ++h) H[h] = Xin[h];
    int c0 = 0;
    if constexpr (kPairArg && P == 1 && NL >= 2) {
      // Cells c and c+1 update different column sums, so once both cells'
      // horizontal prefixes are known their column-sum updates run as paired
      // FP32 instructions (same roundings as the scalar code below).
#pragma unroll
      for (int c = 0; c + 1 < C; c += 2) {
        T h0[NX], h1[NX];
#pragma unroll
        for (int k = 2; k <= NL; ++k) {
          h0[k - 2] = H[k - 2];
          H[k - 2] += Ccol[k - 2][c];
          h1[k - 2] = H[k - 2];
          H[k - 2] += Ccol[k - 2][c + 1];
        }
        const float2 zz = make_float2(Z[c], Z[c + 1]);
        float2 r = __fadd2_rn(make_float2(Ccol[0][c], Ccol[0][c + 1]), zz);
        Ccol[0][c] = r.x;
        Ccol[0][c + 1] = r.y;
#pragma unroll
        for (int k = 2; k < NL; ++k) {
          r = __ffma2_rn(zz, make_float2(h0[k - 2], h1[k - 2]),
                         make_float2(Ccol[k - 1][c], Ccol[k - 1][c + 1]));
          Ccol[k - 1][c] = r.x;
          Ccol[k - 1][c + 1] = r.y;
        }
        r = __ffma2_rn(zz, make_float2(h0[NL - 2], h1[NL - 2]), make_float2(Clast[c], Clast[c + 1]));
        Clast[c] = r.x;
        Clast[c + 1] = r.y;
      }
      c0 = C & ~1;
    }
#pragma unroll
    for (int c = c0; c < C; ++c) {
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
      if (NL >= 2) Clast[c] = fma(z, Hold[NL - 2], Clast[c]);
      else Clast[c] += z;
    }
#pragma unroll
    for (int h = 0; h < NX; ++h) X[h] = H[h];
  }

  // Folds a finished strip's column totals into the lane's level totals: the
  // lane's C column sums of a level are added pairwise in T (depth
  // ceil(log2 C)), the sum once converted and accumulated in FP64.  Lanes
  // reach this at different steps, so it runs for one lane at a time; the
  // short form keeps that serial part small.
  __device__ void end_item() {
#pragma unroll
    for (int k = 1; k < NL; ++k) accd[k] += (double)pair_sum<C>(Ccol[L::off(k + 1)]);
    accd[NL] += (double)pair_sum<C>(Clast);
  }

  // End of a stacked pair at its separator row: fold and publish its level
  // totals (reduction slot `slot`), clear the state for the next pair.
  __device__ void fold_pair(long long slot, int lane) {
    end_item();
    end_task(slot, 0, lane);
    begin_item();
  }

  __device__ void end_task(long long seq, int, int lane) {
#pragma unroll
    for (int k = 1; k <= NL; ++k) {
      red[seq & 1][k - 1][lane] = accd[k];
      accd[k] = 0.0;
    }
  }

  // Warp-wide: sum the 32 lanes' level totals of task t (FP64, fixed order).
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

template <typename T, int KD, int C, int NL, int P, bool DIFF, int WPB, bool EXT>
__global__ void __launch_bounds__(WPB * 32)
dp_fwd_kernel(const SweepArgs<T> args) {
  __shared__ ItemMeta<T> ring[WPB][kItemRing];
  __shared__ double red[WPB][2][NL][32];
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  auto* sm = reinterpret_cast<SweepSmem<T, KD, C>*>(dyn_smem);
  DpPolicy<T, C, NL, P, WPB> pol;
  pol.init(red[threadIdx.x >> 5], args.out, args.ntasks_total, args.nl_out);
  sweep<T, KD, C, DIFF, WPB, EXT>(args, pol, sm[threadIdx.x >> 5], ring[threadIdx.x >> 5]);
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
template <typename T, int C, int F, bool DIFF, bool STK = false>
struct PdePolicy {
  static constexpr int NX = 2 * F;
  static constexpr bool kUnroll2 = C * F <= 16 && sizeof(T) == 4;
  static constexpr bool kPairArg = false;
  // Stacked pairs (SweepArgs::stack_len, the STK instantiations): at a
  // separator row the lane resets its K values to the boundary value 1, on
  // which the separator row (Z = 0) is a no-op that hands on the boundary
  // values (1, 0); each pair's far corner is captured in row() as its cell
  // row comes by.  The stacking checks cost the PDE's light per-cell work
  // 7.6 % on calls that cannot stack (ragged 256 x 256 pairs, L 64-512,
  // dyadic 1: 14.4 -> 15.5 ms), hence kernels of their own.
  static constexpr bool kStack = STK;
  static constexpr bool kCollect = false;
  int slen = 0, tstride = 0;  // stacked sequence length, task stride (nY)
  __device__ void set_stack(int len, int stride) { slen = len; tstride = stride; }
  __device__ void fold_pair(long long, int) { begin_item(); }
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
    // Far corner of the first (or only) pair; a stacked item's later pairs
    // follow slen rows apart (row()).
    tgt_r = slen > 0 ? slen - 2 : lx - 1;
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

  __device__ void row(const T (&Z)[C], const T (&Xin)[NX], bool mask_last, bool valid,
                      int r, const ItemInfo& it, int lane) {
    if (!valid) return;
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
      if (slen > 0) {  // pair r / slen of a stacked item; the next corner
        out[it.task + (r / slen) * tstride] = (double)captured;
        tgt_r += slen;
      } else {
        out[it.task] = (double)captured;
      }
    }
  }
  __device__ void end_item() {}
  __device__ void end_task(long long, int, int) {}
  __device__ void collect(long long, int, int) {}
};

template <typename T, int KD, int C, int F, bool DIFF, int WPB, bool EXT, bool STK = false>
__global__ void __launch_bounds__(WPB * 32)
pde_fwd_kernel(const SweepArgs<T> args) {
  __shared__ ItemMeta<T> ring[WPB][kItemRing];
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  auto* sm = reinterpret_cast<SweepSmem<T, KD, C>*>(dyn_smem);
  PdePolicy<T, C, F, DIFF, STK> pol;
  pol.init(args.out);
  sweep<T, KD, C, DIFF, WPB, EXT>(args, pol, sm[threadIdx.x >> 5], ring[threadIdx.x >> 5]);
}

// ---------------------------------------------------------------------------
// Global alignment kernel (ksig/algorithms.py:453-559), no differencing: the
// "cells" are the grid points, Z carries the static-kernel values M.  In log
// space, with M' = M / (2 - M) and logM = log(max(M', 1e-12)),
//   logK[i,j] = logM[i,j] + LSE(logK[i-1,j], logK[i,j-1], logK[i-1,j-1]),
// logK[-1,-1] = 0 and -inf elsewhere on the boundary; the result is logK at
// the last point pair.  The neighbour pattern is the PDE's at F = 1: the
// left value and the corner come from lane l-1, the upper row stays in the
// lane's registers.
// ---------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ T ga_logm(T m) {
  const T mp = m / (T(2) - m);
  return log(fmax(mp, T(1e-12)));
}

template <typename T>
__device__ __forceinline__ T lse3(T a, T b, T c) {
  const T m = fmax(a, fmax(b, c));
  if (!(m > -INFINITY)) return m;  // all three -inf (or a NaN input)
  return m + log(exp(a - m) + exp(b - m) + exp(c - m));
}

template <typename T, int C>
struct GaPolicy {
  static constexpr int NX = 1;
  static constexpr bool kUnroll2 = false;
  static constexpr bool kPairArg = false;
  static constexpr bool kStack = false;
  static constexpr bool kCollect = false;
  static constexpr int STRIP = 32 * C;
  T X[NX];
  T Kr[C];       // logK of the row above, the lane's columns
  T kcorner;     // logK at the lane's left boundary on the row above
  double* out;
  int tgt_s, tgt_lane, tgt_c, tgt_r;

  __device__ void init(double* out_) {
    out = out_;
    tgt_s = -1; tgt_lane = -1; tgt_c = 0; tgt_r = -1;
    X[0] = T(-INFINITY);
  }
  __device__ void begin_item() {
#pragma unroll
    for (int c = 0; c < C; ++c) Kr[c] = T(-INFINITY);
    kcorner = T(-INFINITY);
  }
  __device__ void begin_task(const ItemInfo& it, int lane) {
    if (lane == 0) kcorner = T(0);  // logK[-1, -1] = log 1
    tgt_r = it.Lx - 1;
    const int col = it.Ly - 1;
    tgt_s = col / STRIP;
    const int rem = col - tgt_s * STRIP;
    tgt_lane = rem / C;
    tgt_c = rem - tgt_lane * C;
  }
  __device__ void left_boundary(T (&Xin)[NX]) { Xin[0] = T(-INFINITY); }

  __device__ void row(const T (&Z)[C], const T (&Xin)[NX], bool, bool valid, int r,
                      const ItemInfo& it, int lane) {
    if (!valid) return;
    T klo = kcorner;
    T kln = Xin[0];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const T up = Kr[c];
      const T v = ga_logm(Z[c]) + lse3(up, kln, klo);
      klo = up;
      kln = v;
      Kr[c] = v;
    }
    X[0] = kln;
    kcorner = Xin[0];
    if (r == tgt_r && it.s == tgt_s && lane == tgt_lane) {
      T captured = T(0);
#pragma unroll
      for (int c = 0; c < C; ++c) captured = (c == tgt_c) ? Kr[c] : captured;
      out[it.task] = (double)captured;
    }
  }
  __device__ void end_item() {}
  __device__ void end_task(long long, int, int) {}
  __device__ void collect(long long, int, int) {}
};

template <typename T, int KD, int C, int WPB>
__global__ void __launch_bounds__(WPB * 32)
ga_fwd_kernel(const SweepArgs<T> args) {
  __shared__ ItemMeta<T> ring[WPB][kItemRing];
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  auto* sm = reinterpret_cast<SweepSmem<T, KD, C>*>(dyn_smem);
  GaPolicy<T, C> pol;
  pol.init(args.out);
  sweep<T, KD, C, false, WPB, false>(args, pol, sm[threadIdx.x >> 5], ring[threadIdx.x >> 5]);
}

}  // namespace ksig
