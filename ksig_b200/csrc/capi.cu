// C ABI of the ksig_b200 library: argument checks, workspace layout, packing
// and kernel dispatch.  Declarations and reference citations live in
// include/ksig_b200.h.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "normalize.cuh"
#include "pack.cuh"
#include "registry.h"
#include "sweep.cuh"
#include "dp_bwd.cuh"
#include "pde_bwd.cuh"
#include "plain.cuh"
#include "gram.cuh"
#include "gram_tc.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace ksig {
namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(KSIG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define KSIG_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

std::atomic<unsigned long long> g_launches{0};

// Optional CUDA-event timing of the main sweep kernels (bench / profiling).
struct Profiler {
  std::mutex mu;
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
};
Profiler& prof() {
  static Profiler p;
  return p;
}

// Dynamic shared memory of a sweep kernel: one staging slot of C packed rows
// per lane (SweepSmem in sweep.cuh).
size_t sweep_dyn_smem_bytes(int wpb, int c, int rs, size_t es) {
  return (size_t)wpb * 32 * c * rs * es;
}

// Raises the kernel's dynamic shared-memory limit once per (device, kernel).
cudaError_t ensure_smem_attr(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<int, const void*>, size_t>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  for (auto& d : done)
    if (d.first.first == dev && d.first.second == func && d.second >= bytes) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done.push_back({{dev, func}, bytes});
  return e;
}

// Launches `func` and, when profiling is on, brackets it with CUDA events on
// the same stream.
cudaError_t launch_main(const void* func, dim3 grid, dim3 block, void** args, size_t smem,
                        cudaStream_t st) {
  Profiler& P = prof();
  std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
  bool timed = false;
  {
    std::lock_guard<std::mutex> lk(P.mu);
    if (P.on) {
      if (!P.pool.empty()) {
        ev = P.pool.back();
        P.pool.pop_back();
      } else {
        cudaEventCreate(&ev.first);
        cudaEventCreate(&ev.second);
      }
      timed = ev.first && ev.second;
    }
  }
  if (timed) cudaEventRecord(ev.first, st);
  cudaError_t e = cudaLaunchKernel(func, grid, block, args, smem, st);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (timed) {
    cudaEventRecord(ev.second, st);
    std::lock_guard<std::mutex> lk(P.mu);
    P.pending.push_back(ev);
  }
  return e;
}

int sm_count() {
  static std::mutex mu;
  static std::vector<int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
  if (cache[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = n;
  }
  return cache[dev];
}

// Finds the best compiled instantiation: exact op/dtype/order/diff, the
// smallest kd >= need_kd, the smallest nl >= need_nl (DP: extra levels are
// computed and dropped), and the column count closest to want_c (prefer the
// largest c <= want_c, else the smallest above).
const KernelEntry* find_kernel(int op, int f64, int need_kd, int want_c, int need_nl,
                               int p, int diff) {
  const KernelEntry* best = nullptr;
  auto better = [&](const KernelEntry& e) {
    if (!best) return true;
    if (e.kd != best->kd) return e.kd < best->kd;
    if (e.nl != best->nl) return e.nl < best->nl;
    const bool eb = e.c <= want_c, bb = best->c <= want_c;
    if (eb != bb) return eb;
    return eb ? e.c > best->c : e.c < best->c;
  };
  for (int t = 0; t < kNumTables; ++t) {
    for (int i = 0; i < kAllTables[t].n; ++i) {
      const KernelEntry& e = kAllTables[t].entries[i];
      if (e.op != op || e.f64 != f64 || e.p != p || e.diff != diff) continue;
      if (e.kd < need_kd || e.nl < need_nl) continue;
      if (better(e)) best = &e;
    }
  }
  return best;
}

size_t align_up(size_t v, size_t a = 256) { return (v + a - 1) / a * a; }

// RBF exponent scale a = log2(e) / max(2 s^2, 1e-12) (ksig/static/kernels.py:
// 258-260 in base 2); 0 for the other kinds.
double rbf_alpha(int kind, double param) {
  return kind == KSIG_STATIC_RBF ? 1.4426950408889634 / fmax(2.0 * param * param, 1e-12) : 0.0;
}

// Workspace carve-up shared by the forward kernels.
struct FwdPlan {
  int family;             // 0 DP, 1 PDE, 2 global alignment
  int f64, kd, rs, c, nl, nl_out, p, diff, nx_exchange;
  long long ntasks;
  int multi, grid, wpb;
  size_t dyn_smem;
  long long rows_max, scratch_per_warp, nwarps;
  int ordered;            // workspace holds a longest-first task order
  size_t sort_tmp;        // radix-sort temporary bytes
  // Gram input (gram.cuh): the call runs in chunks of gram_chunk tasks, each
  // with a [gram_rows][gram_ld] slot of static-kernel values.
  int gin, gram_rows, gram_ld;
  long long gram_chunk, gram_slot;
  size_t off_status, off_xr, off_yr, off_xstart, off_ystart, off_xlen, off_ylen,
      off_okeys, off_okeys2, off_ovals, off_order, off_sort, off_scratch, off_gram, total;
  const KernelEntry* k;
};

// Workspace offsets of the packed points, lengths, starts, the task-order
// buffers and the per-warp scratch (last, so that the adjoint plans can
// re-size it).
void layout_fwd(FwdPlan& pl, int nX, int LX, int nY, int LY) {
  const size_t es = pl.f64 ? 8 : 4;
  size_t off = 0;
  pl.off_status = off; off = align_up(off + 16);
  pl.off_xr = off; off = align_up(off + (size_t)nX * LX * pl.rs * es);
  pl.off_yr = off; off = align_up(off + (size_t)nY * LY * pl.rs * es);
  pl.off_xstart = off; off = align_up(off + (size_t)nX * 8);
  pl.off_ystart = off; off = align_up(off + (size_t)nY * 8);
  pl.off_xlen = off; off = align_up(off + (size_t)nX * 4);
  pl.off_ylen = off; off = align_up(off + (size_t)nY * 4);
  const size_t no = pl.ordered ? (size_t)pl.ntasks * 4 : 0;
  pl.off_okeys = off; off = align_up(off + no);
  pl.off_okeys2 = off; off = align_up(off + no);
  pl.off_ovals = off; off = align_up(off + no);
  pl.off_order = off; off = align_up(off + no);
  pl.off_sort = off; off = align_up(off + (pl.ordered ? pl.sort_tmp : 0));
  pl.off_scratch = off; off = align_up(off + (size_t)pl.nwarps * pl.scratch_per_warp * es);
  pl.off_gram = off;
  if (pl.gin) off = align_up(off + (size_t)pl.gram_chunk * pl.gram_slot * es);
  pl.total = off;
}

int env_int(const char* name, int def);

// ---- longest-first task order for ragged batches --------------------------
// Pairs of a ragged batch differ in cost by up to the product of the length
// ratios.  Sorting the task indices by cell count (descending) and handing
// them out round-robin gives every warp one task of each cost band, so the
// persistent grid drains evenly.  Tasks keep their output slots.

__global__ void order_keys_kernel(int ntasks, int mode, int nY, const int2* list, int nX,
                                  int nYseq, const int32_t* xlen, const int32_t* ylen, int diff,
                                  uint32_t* keys, int32_t* vals) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x) {
    const int2 ab = decode_task(t, mode, nY, list, nullptr);
    uint32_t key = 0;
    if (ab.x >= 0 && ab.x < nX && ab.y >= 0 && ab.y < nYseq) {
      long long a = (long long)xlen[ab.x] - diff, b = (long long)ylen[ab.y] - diff;
      a = a > 0 ? a : 0;
      b = b > 0 ? b : 0;
      const long long c = a * b;
      key = c > 0xffffffffLL ? 0xffffffffu : (uint32_t)c;
    }
    keys[t] = key;
    vals[t] = t;
  }
}

// Decides whether a plan orders its tasks and sizes the sort temporary.
void plan_order(FwdPlan& pl, int pairs_mode) {
  pl.ordered = 0;
  pl.sort_tmp = 0;
  if (pairs_mode == KSIG_PAIRS_DIAG || pl.ntasks < 2048 || !env_int("KSIG_TASK_ORDER", 1)) return;
  size_t bytes = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(
      nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr, (const int32_t*)nullptr,
      (int32_t*)nullptr, (int)pl.ntasks);
  if (e != cudaSuccess) return;
  pl.ordered = 1;
  pl.sort_tmp = bytes;
}

// Builds the order in the workspace (after packing, which wrote the
// lengths); null when the plan has no order or the batch is not ragged.
const int* build_order(const FwdPlan& pl, bool ragged, int mode, int nY, const int32_t* list,
                       int nX, int nYseq, char* ws, cudaStream_t st, int* rc) {
  *rc = KSIG_OK;
  if (!pl.ordered || !ragged) return nullptr;
  uint32_t* k1 = reinterpret_cast<uint32_t*>(ws + pl.off_okeys);
  uint32_t* k2 = reinterpret_cast<uint32_t*>(ws + pl.off_okeys2);
  int32_t* v1 = reinterpret_cast<int32_t*>(ws + pl.off_ovals);
  int32_t* v2 = reinterpret_cast<int32_t*>(ws + pl.off_order);
  const int32_t* xl = reinterpret_cast<const int32_t*>(ws + pl.off_xlen);
  const int32_t* yl = reinterpret_cast<const int32_t*>(ws + pl.off_ylen);
  const int n = (int)pl.ntasks;
  int blocks = (n + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  order_keys_kernel<<<blocks, 256, 0, st>>>(n, mode, nY, reinterpret_cast<const int2*>(list), nX,
                                            nYseq, xl, yl, pl.diff, k1, v1);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    size_t tmp = pl.sort_tmp;
    e = cub::DeviceRadixSort::SortPairsDescending(ws + pl.off_sort, tmp, k1, k2, v1, v2, n, 0, 32,
                                                  st);
  }
  if (e != cudaSuccess) {
    *rc = cuda_fail(e, "task order");
    return nullptr;
  }
  g_launches.fetch_add(2, std::memory_order_relaxed);
  return v2;
}

long long num_pairs(int mode, int nX, int nY, int n_list) {
  switch (mode) {
    case KSIG_PAIRS_FULL: return (long long)nX * nY;
    case KSIG_PAIRS_UPPER: return (long long)nX * (nX + 1) / 2;
    case KSIG_PAIRS_DIAG: return nX;
    case KSIG_PAIRS_LIST: return n_list;
  }
  return -1;
}

// Integer tuning override from the environment (unset -> def).
int env_int(const char* name, int def) {
  const char* v = getenv(name);
  if (!v || !*v) return def;
  return atoi(v);
}

// Column count per lane: smallest c whose strip covers the longest column
// sequence in one strip, capped by what the register budget allows.
// KSIG_FWD_COLS overrides the choice (tuning).
// Column counts chosen by the autotuner per kernel family (0: heuristic).
std::atomic<int> g_tuned_cols[4];

int tuned_cols(int op) { return (op >= 0 && op < 4) ? g_tuned_cols[op].load() : 0; }

int want_cols(int ly_cells, int cap, int op) {
  const int tuned = tuned_cols(op);
  if (tuned > 0) return tuned;
  const int forced = env_int("KSIG_FWD_COLS", 0);
  if (forced > 0) return forced;
  // The PDE and global-alignment sweeps are compiled for 2, 4 and 8
  // columns (8 up to 16 coordinates).  For the PDE the widest strip that
  // covers a row in one pass wins: 512 x 512 pairs of L = 200 ran in
  // 23.7 ms with 8 columns (one strip) against 27.8 ms with 4 (two strips),
  // 33.1 against 37.9 ms at dyadic order 1 (caps per family in plan_fwd).
  static const int opts[] = {2, 4, 8};
  if (op == OP_DP_FWD) {
    // Fewest lane-steps per row with a per-step overhead of 1.5 cells:
    // strips * (C + 1.5), ties to the wider strip.  Fitted to B200 timings
    // of the FP32 order-1 sweep (C = 4 beats C = 7 at 255 columns, C = 7
    // wins at 199 and 399).
    int best = 0;
    long long best_cost = -1;
    for (int c : {2, 4, 7}) {
      if (c > cap) break;
      const long long strip = 32 * c - 1;
      const long long ns = ly_cells <= strip ? 1 : (ly_cells + strip - 1) / strip;
      const long long cost = ns * (2 * c + 3);
      if (best_cost < 0 || cost <= best_cost) { best_cost = cost; best = c; }
    }
    return best > 0 ? best : cap;
  }
  for (int c : opts) {
    if (c > cap) break;
    if (32 * c - 1 >= ly_cells) return c;
  }
  return cap;
}

// family: 0 DP, 1 PDE (order_or_dyadic = dyadic order), 2 global alignment
// (no differencing; order_or_dyadic unused).
// layout_only: the packing and workspace layout without a sweep kernel (the
// plain one-pair-per-block kernels use it; any d, order and n_levels).
int plan_fwd(int family, int nX, int LX, int nY, int LY, int d, int dtype, int n_levels,
             int order_or_dyadic, int difference, int pairs_mode, int n_list,
             FwdPlan& pl, bool allow_order = true, bool ext = false,
             bool layout_only = false) {
  const bool pde = family == 1, ga = family == 2;
  if (dtype != KSIG_DTYPE_F32 && dtype != KSIG_DTYPE_F64)
    return fail(KSIG_ERR_INVALID, "dtype must be KSIG_DTYPE_F32 or KSIG_DTYPE_F64");
  if (nX <= 0 || LX <= 0 || d <= 0) return fail(KSIG_ERR_INVALID, "empty X (n=%d, L=%d, d=%d)", nX, LX, d);
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; }
  else if (nY <= 0 || LY <= 0) return fail(KSIG_ERR_INVALID, "empty Y (n=%d, L=%d)", nY, LY);
  if (pairs_mode < 0 || pairs_mode > KSIG_PAIRS_LIST) return fail(KSIG_ERR_INVALID, "bad pairs_mode %d", pairs_mode);
  const long long np = num_pairs(pairs_mode, nX, nY, n_list);
  if (np < 0 || np > (long long)0x7fffffff) return fail(KSIG_ERR_INVALID, "pair count %lld out of range", np);
  pl = FwdPlan{};
  pl.family = family;
  pl.f64 = dtype == KSIG_DTYPE_F64;
  pl.diff = difference ? 1 : 0;
  pl.ntasks = np;
  int need_nl = 0, p = 0;
  if (ga) {
    pl.diff = 0;
    p = 1;
  } else if (pde) {
    if (order_or_dyadic < 0 || order_or_dyadic > 3)
      return fail(KSIG_ERR_UNSUPPORTED, "dyadic_order %d not in [0, 3]", order_or_dyadic);
    p = 1 << order_or_dyadic;
    need_nl = 0;
  } else {
    if (n_levels <= 0) return fail(KSIG_ERR_INVALID, "n_levels must be positive");
    int ord = order_or_dyadic;
    ord = (ord <= 0 || ord >= n_levels) ? n_levels : ord;  // ksig/algorithms.py:37
    p = ord;
    need_nl = n_levels;
  }
  const int ly_cells = pl.diff ? LY - 1 : LY;
  const int lx_cells = pl.diff ? LX - 1 : LX;
  const int op = ga ? OP_GA_FWD
                   : ext ? (pde ? OP_PDE_FWD_EXT : OP_DP_FWD_EXT) : (pde ? OP_PDE_FWD : OP_DP_FWD);
  // Column caps measured on a B200 (256 x 256 pairs, L = 200, d = 9): the
  // PDE gains from 8 columns up to dyadic order 2 (4.9 against 7.6 ms at
  // order 0, 13.9 against 20.0 ms at order 2); order 3 (C * F = 64 refined
  // values per lane) stays at 4; the global-alignment sweep (a log-sum-exp
  // per cell) ran 21.4 ms with 4 columns and 33.8 ms with 8.
  const int cap = ga ? 4 : (pde && p >= 8) ? 4 : 8;
  const int want = want_cols(ly_cells, cap, op);
  // KSIG_FORCE_GIN=1 takes the Gram-input path even where a register-Gram
  // tile exists (measurement of the two Gram forms on the same shapes).
  const KernelEntry* k = (layout_only || env_int("KSIG_FORCE_GIN", 0))
                             ? nullptr
                             : find_kernel(op, pl.f64, d, want, need_nl, p, pl.diff);
  if (layout_only) {
    pl.k = nullptr;
    pl.kd = round_up(d, 4);
    pl.c = 1;
    pl.nl = need_nl;
    pl.nl_out = need_nl;
    pl.p = p;
    pl.wpb = 1;
    pl.rs = round_up(pl.kd + 1, pl.f64 ? 2 : 4);
    pl.grid = 1;
    pl.nwarps = 0;
    pl.scratch_per_warp = 0;
    if (allow_order) plan_order(pl, pairs_mode);
    layout_fwd(pl, nX, LX, nY, LY);
    return KSIG_OK;
  }
  if (!k && !layout_only) {
    // No register-Gram tile for this shape (e.g. more channels than the
    // widest compiled one): the Gram-input instantiation of the same family
    // with a precomputed Gram (any static kind, any d).
    const int gop = ga ? OP_GA_FWD : (pde ? OP_PDE_FWD : OP_DP_FWD);
    k = find_kernel(gop, pl.f64, 0, want, need_nl, p, pl.diff);
    if (k && k->kd != 0) k = nullptr;
    if (k) pl.gin = 1;
  }
  if (!k)
    return fail(KSIG_ERR_UNSUPPORTED,
                "no compiled %s kernel for dtype=%s d=%d n_levels=%d order/F=%d difference=%d%s",
                ga ? "global-alignment" : pde ? "PDE" : "DP", pl.f64 ? "f64" : "f32", d, n_levels,
                p, pl.diff,
                ext ? " (polynomial / Matern / rational quadratic static kernel)" : "");
  pl.k = k;
  pl.kd = pl.gin ? round_up(d, 4) : k->kd;
  pl.c = k->c;
  pl.nl = k->nl;
  pl.nl_out = need_nl;
  pl.p = p;
  pl.wpb = k->wpb;
  const size_t es = pl.f64 ? 8 : 4;
  pl.rs = round_up(pl.kd + 1, (int)(16 / es));
  const int strip = pl.diff ? 32 * pl.c - 1 : 32 * pl.c;
  pl.multi = ly_cells > strip ? 1 : 0;
  if (ga) {
    pl.nx_exchange = 1;
  } else if (pde) {
    pl.nx_exchange = 2 * p;
  } else {
    int nh = 0;
    for (int q = 2; q <= pl.nl; ++q) nh += q < p ? q : p;
    pl.nx_exchange = nh > 0 ? nh : 1;
  }
  // Grid: one warp per SM slot, never more warps than pairs.
  pl.dyn_smem = sweep_dyn_smem_bytes(k->wpb, pl.c, pl.gin ? 1 : pl.rs, es);
  cudaError_t e = ensure_smem_attr(k->func, pl.dyn_smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k->func, k->wpb * 32, pl.dyn_smem);
  if (e != cudaSuccess || occ <= 0) occ = 1;
  const int sms = sm_count() > 0 ? sm_count() : 148;
  long long warps = (long long)sms * occ * k->wpb;
  if (warps > np) warps = np > 0 ? np : 1;
  pl.grid = (int)((warps + k->wpb - 1) / k->wpb);
  const long long nwarps = (long long)pl.grid * k->wpb;
  pl.rows_max = lx_cells > 32 ? lx_cells : 32;
  pl.scratch_per_warp = pl.multi ? pl.rows_max * pl.nx_exchange : 0;
  pl.nwarps = nwarps;
  if (pl.gin) {
    pl.gram_rows = LX;
    pl.gram_ld = LY;
    pl.gram_slot = (long long)LX * LY;
    const long long budget = (long long)env_int("KSIG_GRAM_MB", 4096) << 20;
    long long chunk = budget / (pl.gram_slot * (long long)es);
    if (chunk < 1) chunk = 1;
    if (chunk > np) chunk = np > 0 ? np : 1;
    if (chunk > 65535) chunk = 65535;  // grid.y of gram_kernel
    pl.gram_chunk = chunk;
  }
  if (allow_order) plan_order(pl, pairs_mode);
  layout_fwd(pl, nX, LX, nY, LY);
  return KSIG_OK;
}

// Re-targets a plan's packing to another kernel's padded width (the
// adjoint kernels are compiled for their own KD set).
void repack_for(FwdPlan& pl, int kd, int nX, int LX, int nY, int LY) {
  pl.kd = kd;
  pl.rs = round_up(kd + 1, pl.f64 ? 2 : 4);
  layout_fwd(pl, nX, LX, nY, LY);
}

__global__ void starts_kernel(int64_t* start, int n, int L) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    start[i] = (int64_t)i * L;
}

template <typename T>
int pack(const void* src, const int32_t* len, int n, int L, int d, int src_f64, int kind,
         double param, int row_side, const FwdPlan& pl, T* dst, int64_t* start,
         int32_t* len_out, int* status, cudaStream_t st) {
  PackArgs a{src, len, n, L, d, src_f64, kind, param, row_side, pl.kd, pl.rs, len_out, status};
  const long long total = (long long)n * L;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  pack_rows_kernel<T><<<blocks, 256, 0, st>>>(a, dst);
  KSIG_CUDA(cudaGetLastError());
  starts_kernel<<<(n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, 256, 0, st>>>(start, n, L);
  KSIG_CUDA(cudaGetLastError());
  g_launches.fetch_add(2, std::memory_order_relaxed);
  return KSIG_OK;
}

template <typename T>
int run_fwd(const FwdPlan& pl, const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
            const int32_t* lenY, int nY, int LY, int d, int src_f64, int kind, double param,
            const StaticParams& sp, int mode, const int32_t* list, double* out, char* ws,
            cudaStream_t st) {
  int* status = reinterpret_cast<int*>(ws + pl.off_status);
  T* xr = reinterpret_cast<T*>(ws + pl.off_xr);
  T* yr = reinterpret_cast<T*>(ws + pl.off_yr);
  int64_t* xs = reinterpret_cast<int64_t*>(ws + pl.off_xstart);
  int64_t* ys = reinterpret_cast<int64_t*>(ws + pl.off_ystart);
  int32_t* xl = reinterpret_cast<int32_t*>(ws + pl.off_xlen);
  int32_t* yl = reinterpret_cast<int32_t*>(ws + pl.off_ylen);
  const bool self = mode == KSIG_PAIRS_UPPER || mode == KSIG_PAIRS_DIAG;
  int rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 1, pl, xr, xs, xl, status, st);
  if (rc) return rc;
  if (self) rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  else rc = pack<T>(Y, lenY, nY, LY, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  if (rc) return rc;
  SweepArgs<T> a{};
  a.xr = xr; a.xstart = xs; a.xlen = xl;
  a.yr = yr; a.ystart = ys; a.ylen = yl;
  a.mode = mode;
  a.nY = self ? nX : nY;
  a.list = reinterpret_cast<const int2*>(list);
  a.order = build_order(pl, lenX || lenY, mode, self ? nX : nY, list, nX, self ? nX : nY, ws, st,
                        &rc);
  if (rc) return rc;
  a.ntasks = (int)pl.ntasks;
  a.ntasks_total = (int)pl.ntasks;
  a.task_base = 0;
  // Row prefetch distance (steps ahead): the Gram-input sweeps read a new
  // slot row every step in every lane (4 steps: 4 % faster on B200); the
  // register-Gram sweeps gained nothing from it.
  a.x_prefetch = env_int("KSIG_XPF", pl.gin ? 4 : 0);
  // Column-major blocks per warp (sweep.cuh, SweepArgs::visit_per) where the
  // pairs are a full grid or the upper triangle of K(X) over equal-length
  // sequences: consecutive pairs of a
  // warp then share their column sequence, a pair switch reloads no column
  // points, and every warp gets the same number of equal pairs (512 x 512
  // pairs, L = 200, d = 9, m = 5 on a B200: 24.4 -> 23.3 ms).  Ragged grids
  // keep the round-robin order over the longest-first permutation.
  // KSIG_VISIT=0 keeps the round-robin order (measurement).
  a.visit_per = 0;
  if (!pl.gin && (mode == KSIG_PAIRS_FULL || mode == KSIG_PAIRS_UPPER) && !a.order && !lenX &&
      !lenY && env_int("KSIG_VISIT", 1) > 0) {
    const long long nw = (long long)pl.grid * pl.k->wpb;
    a.visit_per = (pl.ntasks + nw - 1) / nw;
  }
  // Stacked pairs (SweepArgs::stack_len): the pairs of one column in a
  // warp's block run as one item, the separator rows between the stacked
  // row sequences folding each pair (DP levels) or resetting the lane's K
  // values (PDE), so a column needs one item switch instead of one per
  // pair.  An item switch costs the warp about 35 steps at three times the
  // cost of a plain step, the stacked form a few instructions per step.
  // B200, 512 columns of L = 200, d = 9, DP m = 5: 512 rows of L = 200
  // 20.7 -> 16.7 ms, 256 of L = 400 17.7 -> 16.2 ms, 64 of L = 1600
  // 15.5 -> 16.0 ms; hence row sequences up to 1024 points.  KSIG_STACK=0
  // switches it off, KSIG_STACK=1 on for any length.
  a.stack_len = 0;
  {
    const int st = env_int("KSIG_STACK", -1);
    if (a.visit_per > 0 && mode == KSIG_PAIRS_FULL && (pl.family == 0 || pl.family == 1) &&
        pl.diff && !pl.multi && LX >= 17 && (st > 0 || (st < 0 && LX <= 1024)))
      a.stack_len = LX;
  }
  // PDE: stacked pairs run in kernels of their own (OP_PDE_FWD_STACK, the
  // same tile); without one the call does not stack.  Column-major blocks
  // without stacking: 24.1 -> 21.6 ms with one strip per pair (512 x 512
  // pairs, L = 200, 8 columns), but 1-3 % slower with two strips (4
  // columns), where every strip reloads its column points anyway.
  const void* func = pl.k->func;
  if (pl.family == 1 && pl.k->op != OP_PDE_FWD) a.stack_len = 0;  // EXT kinds: no stacked tiles
  if (pl.family == 1 && a.stack_len > 0) {
    const KernelEntry* ks = find_kernel(OP_PDE_FWD_STACK, pl.f64, pl.k->kd, pl.c, 0, pl.p, 1);
    if (ks && ks->kd == pl.k->kd && ks->c == pl.c && ks->p == pl.p && ks->wpb == pl.k->wpb &&
        ensure_smem_attr(ks->func, pl.dyn_smem) == cudaSuccess)
      func = ks->func;
    else
      a.stack_len = 0;
  }
  if (pl.family == 1 && a.stack_len == 0 && pl.multi) a.visit_per = 0;
  a.kind = kind;
  a.sp = sp;
  a.ralpha = (T)rbf_alpha(kind, param);
  a.out = out;
  a.scratch = pl.multi ? reinterpret_cast<T*>(ws + pl.off_scratch) : nullptr;
  a.scratch_per_warp = pl.scratch_per_warp;
  a.multi_strip = pl.multi;
  a.nl_out = pl.nl_out;
  a.nX = nX;
  a.nYseq = self ? nX : nY;
  a.status = status;
  void* kargs[] = {&a};
  if (!pl.gin) {
    KSIG_CUDA(launch_main(func, dim3(pl.grid), dim3(pl.k->wpb * 32), kargs, pl.dyn_smem, st));
    return KSIG_OK;
  }
  // Gram input: per chunk of tasks, the Gram slots, then the sweep on them.
  GramArgs<T> g{};
  g.xr = xr; g.xstart = xs; g.xlen = xl; g.yr = yr; g.ystart = ys; g.ylen = yl;
  g.rs = pl.rs; g.kd = pl.kd;
  g.mode = mode; g.nY = a.nY; g.list = a.list; g.order = a.order;
  g.nX = nX; g.nYseq = a.nYseq;
  g.kind = kind; g.ralpha = a.ralpha; g.sp = sp;
  g.gram = reinterpret_cast<T*>(ws + pl.off_gram);
  g.slot = pl.gram_slot; g.ld = pl.gram_ld;
  // The CUDA-core difference tiles (gram.cuh) by default; RBF in FP32 with
  // KSIG_GRAM_TC=1: the tensor-core tiles (gram_tc.cuh).  The tensor-core
  // tiles are faster from 128 coordinates (B200, 128 x 128 pairs, L = 200:
  // 15.1 vs 16.8 ms at d = 128, 25.7 vs 31.2 ms at d = 256), but with one
  // centre per 32 columns and 3xTF32 products they missed the 1e-5 bar on
  // widely spread paths (d = 64 and d = 160 walks with steps of 0.2 per
  // channel), where the difference tiles do not cancel.
  bool tc = false;
  if constexpr (std::is_same<T, float>::value)
    tc = kind == KIND_RBF && env_int("KSIG_GRAM_TC", 0) > 0;
  const int tm = tc ? kTcM : kGramTile, tn = tc ? kTcN : kGramTile;
  const int tiles_x = (pl.gram_rows + tm - 1) / tm;
  g.tiles_y = (pl.gram_ld + tn - 1) / tn;
  g.status = status;
  if constexpr (std::is_same<T, float>::value) {
    if (tc) {
      cudaError_t ce = ensure_smem_attr((const void*)&gram_tc_kernel, gram_tc_smem_bytes());
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaFuncSetAttribute(gram_tc_kernel)");
    }
  }
  a.gram = g.gram; a.gram_slot = pl.gram_slot; a.gram_ld = pl.gram_ld;
  for (long long t0 = 0; t0 < pl.ntasks; t0 += pl.gram_chunk) {
    const long long nt = pl.ntasks - t0 < pl.gram_chunk ? pl.ntasks - t0 : pl.gram_chunk;
    g.task_base = (int)t0; g.ntasks = (int)nt;
    const dim3 ggrid(tiles_x * g.tiles_y, (unsigned)nt);
    if constexpr (std::is_same<T, float>::value) {
      if (tc) {
        void* gargs[] = {&g};
        KSIG_CUDA(launch_main((const void*)&gram_tc_kernel, ggrid, dim3(128), gargs,
                              gram_tc_smem_bytes(), st));
      } else {
        gram_kernel<T><<<ggrid, 256, 0, st>>>(g);
        g_launches.fetch_add(1, std::memory_order_relaxed);
      }
    } else {
      gram_kernel<T><<<ggrid, 256, 0, st>>>(g);
      g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    a.task_base = (int)t0; a.ntasks = (int)nt;
    const long long blocks = (nt + pl.k->wpb - 1) / pl.k->wpb;
    const int grid = blocks < pl.grid ? (int)blocks : pl.grid;
    KSIG_CUDA(launch_main(pl.k->func, dim3(grid), dim3(pl.k->wpb * 32), kargs, pl.dyn_smem, st));
  }
  return KSIG_OK;
}

// Backward: the forward's packing layout plus per-warp scratch for strip
// carries and per-strip column sums (dp_bwd.cuh).
struct BwdPlan {
  FwdPlan f;
  const KernelEntry* k;
  int c, nx, ns_max, rows_max, grid;
  size_t dyn_smem;
  long long scratch_per_warp;
  size_t off_scratch, total;
  long long rec_per_pair;  // split pass: record elements kept per pair
  int ckpt;                // strip checkpointing (dp_bwd.cuh, DpBwdArgs::ckpt)
  const KernelEntry* kc;   // its kernel (dp_bwd_ckpt_kernel), when ckpt
};

int plan_bwd(int nX, int LX, int nY, int LY, int d, int dtype, int n_levels, int order,
             int difference, int pairs_mode, int n_list, BwdPlan& bp, bool allow_ckpt = true) {
  int rc = plan_fwd(false, nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode,
                    n_list, bp.f);
  if (rc) return rc;
  if (!difference)
    return fail(KSIG_ERR_UNSUPPORTED, "gradients need difference=True");
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; }
  const int ly = LY - 1, lx = LX - 1;
  // Column count: fewest lane-steps per row, ns(C) * C, over the compiled
  // variants (ties go to the wider strip: fewer strips, fewer records).
  const int forced = tuned_cols(OP_DP_BWD) > 0 ? tuned_cols(OP_DP_BWD)
                                              : env_int("KSIG_BWD_COLS", 0);
  const KernelEntry* k = nullptr;
  long long best_cost = -1;
  for (int want : {8, 7, 6, 5, 4, 3, 2, 1}) {
    if (forced > 0 && want != forced) continue;
    const KernelEntry* e = find_kernel(OP_DP_BWD, bp.f.f64, d, want, n_levels, bp.f.p, 1);
    if (!e || e->c != want) continue;
    const int strip = 32 * e->c - 1;
    const long long ns = ly <= strip ? 1 : (ly + strip - 1) / strip;
    const long long cost = ns * e->c;
    if (best_cost < 0 || cost < best_cost) { best_cost = cost; k = e; }
  }
  if (!k && forced > 0)
    k = find_kernel(OP_DP_BWD, bp.f.f64, d, forced, n_levels, bp.f.p, 1);
  if (!k)
    return fail(KSIG_ERR_UNSUPPORTED, "no compiled DP backward kernel for dtype=%s d=%d "
                "n_levels=%d order=%d", bp.f.f64 ? "f64" : "f32", d, n_levels, bp.f.p);
  bp.k = k;
  bp.c = k->c;
  repack_for(bp.f, k->kd, nX, LX, nY, LY);
  int nh = 0;
  for (int q = 2; q <= k->nl; ++q) nh += q < bp.f.p ? q : bp.f.p;
  bp.nx = nh > 0 ? nh : 1;
  const int strip = 32 * bp.c - 1;
  bp.ns_max = ly <= strip ? 1 : (ly + strip - 1) / strip;
  bp.rows_max = lx > 1 ? lx : 1;
  const size_t es = bp.f.f64 ? 8 : 4;
  bp.dyn_smem = dp_bwd_smem_bytes(k->wpb, bp.c, bp.f.rs, es);
  cudaError_t e = ensure_smem_attr(k->func, bp.dyn_smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(dp backward)");
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k->func, k->wpb * 32, bp.dyn_smem);
  if (e != cudaSuccess || occ <= 0) occ = 1;
  const int sms = sm_count() > 0 ? sm_count() : 148;
  long long warps = (long long)sms * occ * k->wpb;
  if (warps > bp.f.ntasks) warps = bp.f.ntasks > 0 ? bp.f.ntasks : 1;
  bp.scratch_per_warp = dp_bwd_scratch_elems(bp.ns_max, bp.rows_max, bp.nx, bp.c);
  // Records + final column sums of one pair (the REC and CS regions of the
  // per-warp scratch), padded to 16 bytes.
  bp.rec_per_pair = ((long long)bp.ns_max * (bp.rows_max + 33) * bp.nx * 32 +
                     (long long)bp.ns_max * bp.nx * bp.c * 32 + 3) / 4 * 4;
  // The per-step records grow with the strip count and the row count; keep
  // the whole scratch within a bounded budget.  When the records of every
  // strip would cap the warps below half of what the SMs hold, the adjoint
  // keeps one strip of records and recomputes each strip's from its
  // checkpoint (KSIG_DP_BWD_CKPT: 1 always for multi-strip shapes, 0 never,
  // unset: that rule).  Recomputing costs a second forward pass over those
  // strips: on the 2048-pair ragged order-2 sample (L up to 1024) the
  // workspace fell from 32 GB to 3.3 GB and the adjoint rose 18 % on B200,
  // so a mildly capped grid keeps the full records.
  const long long budget = (long long)env_int("KSIG_DP_BWD_SCRATCH_MB", 32768) << 20;
  long long cap = budget / (long long)(bp.scratch_per_warp * es);
  bp.ckpt = 0;
  const int ck_env = env_int("KSIG_DP_BWD_CKPT", -1);
  bp.kc = nullptr;
  if (allow_ckpt && bp.ns_max > 1 && (ck_env == 1 || (ck_env < 0 && 2 * cap < warps))) {
    const KernelEntry* kc =
        find_kernel(OP_DP_BWD_CKPT, bp.f.f64, k->kd, bp.c, k->nl, bp.f.p, 1);
    if (kc && kc->kd == k->kd && kc->c == bp.c && kc->nl == k->nl) {
      e = ensure_smem_attr(kc->func, bp.dyn_smem);
      if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(dp backward, checkpointed)");
      int occc = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occc, kc->func, k->wpb * 32, bp.dyn_smem);
      if (e != cudaSuccess || occc <= 0) occc = 1;
      warps = (long long)sms * occc * k->wpb;
      if (warps > bp.f.ntasks) warps = bp.f.ntasks > 0 ? bp.f.ntasks : 1;
      bp.ckpt = 1;
      bp.kc = kc;
      bp.scratch_per_warp = dp_bwd_scratch_elems(bp.ns_max, bp.rows_max, bp.nx, bp.c, 1);
      cap = budget / (long long)(bp.scratch_per_warp * es);
    }
  }
  if (warps > cap) warps = cap > (long long)k->wpb ? cap : k->wpb;
  bp.grid = (int)((warps + k->wpb - 1) / k->wpb);
  bp.off_scratch = bp.f.off_scratch;  // the forward scratch region is unused here
  bp.total = align_up(bp.off_scratch + (size_t)bp.grid * k->wpb * bp.scratch_per_warp * es);
  if (bp.total < bp.f.total) bp.total = bp.f.total;
  return KSIG_OK;
}

// The split forward pass compiled for the same tile as the plan's adjoint.
const KernelEntry* rec_fwd_entry(const BwdPlan& bp) {
  const KernelEntry* e = find_kernel(OP_DP_REC_FWD, bp.f.f64, bp.k->kd, bp.c, bp.k->nl, 1, 1);
  if (!e || e->kd != bp.k->kd || e->c != bp.c || e->nl != bp.k->nl) return nullptr;
  return e;
}

template <typename T>
int run_bwd(const BwdPlan& bp, const void* X, const int32_t* lenX, int nX, int LX,
            const void* Y, const int32_t* lenY, int nY, int LY, int d, int src_f64, int kind,
            double param, int mode, const int32_t* list, const double* glev, int nl_out,
            void* dX, double* dparam, char* ws, cudaStream_t st, int phases = 3,
            double* lev = nullptr) {
  const FwdPlan& pl = bp.f;
  int* status = reinterpret_cast<int*>(ws + pl.off_status);
  T* xr = reinterpret_cast<T*>(ws + pl.off_xr);
  T* yr = reinterpret_cast<T*>(ws + pl.off_yr);
  int64_t* xs = reinterpret_cast<int64_t*>(ws + pl.off_xstart);
  int64_t* ys = reinterpret_cast<int64_t*>(ws + pl.off_ystart);
  int32_t* xl = reinterpret_cast<int32_t*>(ws + pl.off_xlen);
  int32_t* yl = reinterpret_cast<int32_t*>(ws + pl.off_ylen);
  const bool self = mode == KSIG_PAIRS_UPPER || mode == KSIG_PAIRS_DIAG;
  int rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 1, pl, xr, xs, xl, status, st);
  if (rc) return rc;
  if (self) rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  else rc = pack<T>(Y, lenY, nY, LY, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  if (rc) return rc;
  DpBwdArgs<T> a{};
  a.xr = xr; a.xstart = xs; a.xlen = xl;
  a.yr = yr; a.ystart = ys; a.ylen = yl;
  a.mode = mode;
  a.nY = self ? nX : nY;
  a.list = reinterpret_cast<const int2*>(list);
  a.order = build_order(pl, lenX || lenY, mode, self ? nX : nY, list, nX, self ? nX : nY, ws, st,
                        &rc);
  if (rc) return rc;
  a.ntasks = (int)pl.ntasks;
  a.nX = nX;
  a.nYseq = self ? nX : nY;
  a.kind = kind;
  a.param = param;
  a.glev = glev;
  a.nl_out = nl_out;
  a.dX = reinterpret_cast<T*>(dX);
  a.LX = LX;
  a.d = d;
  a.dparam = dparam;
  a.scratch = reinterpret_cast<T*>(ws + bp.off_scratch);
  a.scratch_per_warp = bp.scratch_per_warp;
  a.ns_max = bp.ns_max;
  a.rows_max = bp.rows_max;
  a.status = status;
  a.phases = phases;
  a.ckpt = bp.ckpt;
  if (phases != 3) {  // split pass: records per pair, after the plan's regions
    a.rec = reinterpret_cast<T*>(ws + bp.total);
    a.rec_per_pair = bp.rec_per_pair;
  }
  a.lev = lev;
  const void* func = bp.ckpt && phases == 3 ? bp.kc->func : bp.k->func;
  if (phases == 1) {
    const KernelEntry* e = rec_fwd_entry(bp);
    if (!e) return fail(KSIG_ERR_UNSUPPORTED, "no compiled split forward pass for this tile");
    cudaError_t ce = ensure_smem_attr(e->func, bp.dyn_smem);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaFuncSetAttribute(split forward pass)");
    func = e->func;
  }
  void* kargs[] = {&a};
  KSIG_CUDA(launch_main(func, dim3(bp.grid), dim3(bp.k->wpb * 32), kargs, bp.dyn_smem, st));
  return KSIG_OK;
}

// PDE backward: the forward's packing layout plus, per warp, the reversed
// adjoint grid G (refined rows x refined columns) and a strip boundary
// buffer (pde_bwd.cuh).
struct PdeBwdPlan {
  FwdPlan f;
  const KernelEntry* k;
  int c, F, grid, rows_max, ns_max;
  size_t dyn_smem;
  long long scratch_per_warp;
  size_t off_scratch, total;
};

int plan_pde_bwd(int nX, int LX, int nY, int LY, int d, int dtype, int dyadic, int difference,
                 int pairs_mode, int n_list, PdeBwdPlan& bp) {
  int rc = plan_fwd(true, nX, LX, nY, LY, d, dtype, 0, dyadic, difference, pairs_mode, n_list,
                    bp.f);
  if (rc) return rc;
  if (!difference) return fail(KSIG_ERR_UNSUPPORTED, "gradients need difference=True");
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; }
  const int ly = LY - 1, lx = LX - 1;
  bp.F = 1 << dyadic;
  // Column count: fewest lane-steps per row, ns(C) * C, over the compiled
  // variants (ties go to the wider strip: fewer strips, fewer records).
  const int forced = tuned_cols(OP_PDE_BWD) > 0 ? tuned_cols(OP_PDE_BWD)
                                               : env_int("KSIG_BWD_COLS", 0);
  const KernelEntry* k = nullptr;
  long long best_cost = -1;
  for (int want : {8, 4, 2, 1}) {
    if (forced > 0 && want != forced) continue;
    const KernelEntry* e = find_kernel(OP_PDE_BWD, bp.f.f64, d, want, 0, bp.F, 1);
    if (!e || e->c != want) continue;
    const int strip = 32 * e->c - 1;
    const long long ns = ly <= strip ? 1 : (ly + strip - 1) / strip;
    const long long cost = ns * e->c;
    if (best_cost < 0 || cost < best_cost) { best_cost = cost; k = e; }
  }
  if (!k && forced > 0) k = find_kernel(OP_PDE_BWD, bp.f.f64, d, forced, 0, bp.F, 1);
  if (!k)
    return fail(KSIG_ERR_UNSUPPORTED, "no compiled PDE backward kernel for dtype=%s d=%d "
                "dyadic_order=%d", bp.f.f64 ? "f64" : "f32", d, dyadic);
  bp.k = k;
  bp.c = k->c;
  repack_for(bp.f, k->kd, nX, LX, nY, LY);
  bp.rows_max = lx > 1 ? lx : 1;
  const int strip = 32 * bp.c - 1;
  bp.ns_max = ly <= strip ? 1 : (ly + strip - 1) / strip;
  bp.scratch_per_warp = (pde_bwd_scratch_elems(bp.ns_max, bp.rows_max, bp.c, bp.F) + 3) / 4 * 4;
  const size_t es = bp.f.f64 ? 8 : 4;
  bp.dyn_smem = pde_bwd_smem_bytes(k->wpb, bp.c, bp.F, es);
  cudaError_t e = ensure_smem_attr(k->func, bp.dyn_smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(pde backward)");
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k->func, k->wpb * 32, bp.dyn_smem);
  if (e != cudaSuccess || occ <= 0) occ = 1;
  const int sms = sm_count() > 0 ? sm_count() : 148;
  long long warps = (long long)sms * occ * k->wpb;
  // The records grow with rows x strips; keep the scratch within a budget.
  const long long budget = (long long)env_int("KSIG_PDE_BWD_SCRATCH_MB", 16384) << 20;
  const long long cap = budget / (long long)(bp.scratch_per_warp * es);
  if (warps > cap) warps = cap > (long long)k->wpb ? cap : k->wpb;
  if (warps > bp.f.ntasks) warps = bp.f.ntasks > 0 ? bp.f.ntasks : 1;
  bp.grid = (int)((warps + k->wpb - 1) / k->wpb);
  bp.off_scratch = bp.f.off_scratch;
  bp.total = align_up(bp.off_scratch + (size_t)bp.grid * k->wpb * bp.scratch_per_warp * es);
  if (bp.total < bp.f.total) bp.total = bp.f.total;
  return KSIG_OK;
}

template <typename T>
int run_pde_bwd(const PdeBwdPlan& bp, const void* X, const int32_t* lenX, int nX, int LX,
                const void* Y, const int32_t* lenY, int nY, int LY, int d, int src_f64,
                int kind, double param, int mode, const int32_t* list, const double* grad,
                void* dX, double* dparam, char* ws, cudaStream_t st) {
  const FwdPlan& pl = bp.f;
  int* status = reinterpret_cast<int*>(ws + pl.off_status);
  T* xr = reinterpret_cast<T*>(ws + pl.off_xr);
  T* yr = reinterpret_cast<T*>(ws + pl.off_yr);
  int64_t* xs = reinterpret_cast<int64_t*>(ws + pl.off_xstart);
  int64_t* ys = reinterpret_cast<int64_t*>(ws + pl.off_ystart);
  int32_t* xl = reinterpret_cast<int32_t*>(ws + pl.off_xlen);
  int32_t* yl = reinterpret_cast<int32_t*>(ws + pl.off_ylen);
  const bool self = mode == KSIG_PAIRS_UPPER || mode == KSIG_PAIRS_DIAG;
  int rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 1, pl, xr, xs, xl, status, st);
  if (rc) return rc;
  if (self) rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  else rc = pack<T>(Y, lenY, nY, LY, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  if (rc) return rc;
  PdeBwdArgs<T> a{};
  a.xr = xr; a.xstart = xs; a.xlen = xl;
  a.yr = yr; a.ystart = ys; a.ylen = yl;
  a.mode = mode;
  a.nY = self ? nX : nY;
  a.list = reinterpret_cast<const int2*>(list);
  a.order = build_order(pl, lenX || lenY, mode, self ? nX : nY, list, nX, self ? nX : nY, ws, st,
                        &rc);
  if (rc) return rc;
  a.ntasks = (int)pl.ntasks;
  a.nX = nX;
  a.nYseq = self ? nX : nY;
  a.kind = kind;
  a.param = param;
  a.grad = grad;
  a.dX = reinterpret_cast<T*>(dX);
  a.LX = LX;
  a.d = d;
  a.dparam = dparam;
  a.scratch = reinterpret_cast<T*>(ws + bp.off_scratch);
  a.scratch_per_warp = bp.scratch_per_warp;
  a.ns_max = bp.ns_max;
  a.rows_max = bp.rows_max;
  a.status = status;
  void* kargs[] = {&a};
  KSIG_CUDA(launch_main(bp.k->func, dim3(bp.grid), dim3(bp.k->wpb * 32), kargs, bp.dyn_smem, st));
  return KSIG_OK;
}

// Plain one-pair-per-block baseline: the forward packing plus per-CTA
// scratch for Z, one temporary and two sets of p^2 level-state arrays.
struct PlainPlan {
  FwdPlan f;
  int grid, order;
  long long cap;
  size_t off_scratch, total;
};

int plan_plain(int nX, int LX, int nY, int LY, int d, int dtype, int n_levels, int order,
               int pairs_mode, int n_list, PlainPlan& pp) {
  int rc = plan_fwd(false, nX, LX, nY, LY, d, dtype, n_levels, order, 1, pairs_mode, n_list,
                    pp.f, false, false, true);
  if (rc) return rc;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; }
  pp.order = pp.f.p;
  const long long lx = LX > 1 ? LX - 1 : 1, ly = LY > 1 ? LY - 1 : 1;
  pp.cap = lx * ly;
  const size_t es = pp.f.f64 ? 8 : 4;
  const long long per_cta = pp.cap * (2 + 2LL * pp.order * pp.order) * (long long)es;
  const int sms = sm_count() > 0 ? sm_count() : 148;
  long long grid = (long long)sms * 4;
  const long long budget = (long long)env_int("KSIG_PLAIN_SCRATCH_MB", 8192) << 20;
  if (grid * per_cta > budget) grid = budget / per_cta > 1 ? budget / per_cta : 1;
  if (grid > pp.f.ntasks) grid = pp.f.ntasks > 0 ? pp.f.ntasks : 1;
  pp.grid = (int)grid;
  pp.off_scratch = pp.f.off_scratch;
  pp.total = align_up(pp.off_scratch + (size_t)grid * per_cta);
  if (pp.total < pp.f.total) pp.total = pp.f.total;
  return KSIG_OK;
}

template <typename T>
int run_plain(const PlainPlan& pp, const void* X, const int32_t* lenX, int nX, int LX,
              const void* Y, const int32_t* lenY, int nY, int LY, int d, int src_f64, int kind,
              double param, int n_levels, int mode, const int32_t* list, double* out, char* ws,
              cudaStream_t st) {
  const FwdPlan& pl = pp.f;
  int* status = reinterpret_cast<int*>(ws + pl.off_status);
  T* xr = reinterpret_cast<T*>(ws + pl.off_xr);
  T* yr = reinterpret_cast<T*>(ws + pl.off_yr);
  int64_t* xs = reinterpret_cast<int64_t*>(ws + pl.off_xstart);
  int64_t* ys = reinterpret_cast<int64_t*>(ws + pl.off_ystart);
  int32_t* xl = reinterpret_cast<int32_t*>(ws + pl.off_xlen);
  int32_t* yl = reinterpret_cast<int32_t*>(ws + pl.off_ylen);
  const bool self = mode == KSIG_PAIRS_UPPER || mode == KSIG_PAIRS_DIAG;
  int rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 1, pl, xr, xs, xl, status, st);
  if (rc) return rc;
  if (self) rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  else rc = pack<T>(Y, lenY, nY, LY, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  if (rc) return rc;
  PlainArgs<T> a{};
  a.xr = xr; a.xstart = xs; a.xlen = xl; a.yr = yr; a.ystart = ys; a.ylen = yl;
  a.rs = pl.rs; a.kd = pl.kd;
  a.mode = mode; a.nY = self ? nX : nY;
  a.list = reinterpret_cast<const int2*>(list);
  a.ntasks = (int)pl.ntasks; a.nX = nX; a.nYseq = self ? nX : nY;
  a.kind = kind; a.n_levels = n_levels; a.order = pp.order;
  a.ralpha = (T)rbf_alpha(kind, param);
  a.out = out;
  a.scratch = reinterpret_cast<T*>(ws + pp.off_scratch);
  a.cap = pp.cap;
  a.status = status;
  void* kargs[] = {&a};
  KSIG_CUDA(launch_main((const void*)&plain_dp_kernel<T>, dim3(pp.grid), dim3(256), kargs, 0, st));
  return KSIG_OK;
}

// Plain one-pair-per-block adjoint baseline: per-CTA scratch for Z, all
// level states, two sets of p^2 adjoint states, Zbar, one temporary and the
// grid weights, each of LX * LY elements.
struct PlainBwdPlan {
  PlainPlan pp;
  int nbuf;
};

int plan_plain_bwd(int nX, int LX, int nY, int LY, int d, int dtype, int n_levels, int order,
                   int pairs_mode, int n_list, PlainBwdPlan& bp) {
  int rc = plan_plain(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, bp.pp);
  if (rc) return rc;
  PlainPlan& pp = bp.pp;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; }
  const int p = pp.order;
  int states = 0;
  for (int k = 1; k <= n_levels; ++k) { const int f = k < p ? k : p; states += f * f; }
  bp.nbuf = 1 + states + 2 * p * p + 3;
  pp.cap = (long long)(LX > 1 ? LX : 1) * (LY > 1 ? LY : 1);
  const size_t es = pp.f.f64 ? 8 : 4;
  const long long per_cta = pp.cap * bp.nbuf * (long long)es;
  const int sms = sm_count() > 0 ? sm_count() : 148;
  long long grid = (long long)sms * 4;
  const long long budget = (long long)env_int("KSIG_PLAIN_SCRATCH_MB", 8192) << 20;
  if (grid * per_cta > budget) grid = budget / per_cta > 1 ? budget / per_cta : 1;
  if (grid > pp.f.ntasks) grid = pp.f.ntasks > 0 ? pp.f.ntasks : 1;
  pp.grid = (int)grid;
  pp.total = align_up(pp.off_scratch + (size_t)grid * per_cta);
  if (pp.total < pp.f.total) pp.total = pp.f.total;
  return KSIG_OK;
}

template <typename T>
int run_plain_bwd(const PlainBwdPlan& bp, const void* X, const int32_t* lenX, int nX, int LX,
                  const void* Y, const int32_t* lenY, int nY, int LY, int d, int src_f64,
                  int kind, double param, int n_levels, int mode, const int32_t* list,
                  const double* glev, int nl_out, void* dX, double* dparam, char* ws,
                  cudaStream_t st) {
  const PlainPlan& pp = bp.pp;
  const FwdPlan& pl = pp.f;
  int* status = reinterpret_cast<int*>(ws + pl.off_status);
  T* xr = reinterpret_cast<T*>(ws + pl.off_xr);
  T* yr = reinterpret_cast<T*>(ws + pl.off_yr);
  int64_t* xs = reinterpret_cast<int64_t*>(ws + pl.off_xstart);
  int64_t* ys = reinterpret_cast<int64_t*>(ws + pl.off_ystart);
  int32_t* xl = reinterpret_cast<int32_t*>(ws + pl.off_xlen);
  int32_t* yl = reinterpret_cast<int32_t*>(ws + pl.off_ylen);
  const bool self = mode == KSIG_PAIRS_UPPER || mode == KSIG_PAIRS_DIAG;
  int rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 1, pl, xr, xs, xl, status, st);
  if (rc) return rc;
  if (self) rc = pack<T>(X, lenX, nX, LX, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  else rc = pack<T>(Y, lenY, nY, LY, d, src_f64, kind, param, 0, pl, yr, ys, yl, status, st);
  if (rc) return rc;
  PlainBwdArgs<T> a{};
  PlainArgs<T>& f = a.f;
  f.xr = xr; f.xstart = xs; f.xlen = xl; f.yr = yr; f.ystart = ys; f.ylen = yl;
  f.rs = pl.rs; f.kd = pl.kd;
  f.mode = mode; f.nY = self ? nX : nY;
  f.list = reinterpret_cast<const int2*>(list);
  f.ntasks = (int)pl.ntasks; f.nX = nX; f.nYseq = self ? nX : nY;
  f.kind = kind; f.n_levels = n_levels; f.order = pp.order;
  f.ralpha = (T)rbf_alpha(kind, param);
  f.out = nullptr;
  f.scratch = reinterpret_cast<T*>(ws + pp.off_scratch);
  f.cap = pp.cap;
  f.status = status;
  a.glev = glev;
  a.nl_out = nl_out;
  a.dX = reinterpret_cast<T*>(dX);
  a.LX = LX;
  a.d = d;
  a.param = param;
  a.dparam = dparam;
  a.nbuf = bp.nbuf;
  void* kargs[] = {&a};
  KSIG_CUDA(launch_main((const void*)&plain_dp_bwd_kernel<T>, dim3(pp.grid), dim3(256), kargs,
                        0, st));
  return KSIG_OK;
}

// Validates the parameters of any static kernel kind (ksig/utils.py:23-35
// messages) and forms its epilogue constants (common.cuh, static_value).
int static_params(int kind, const double* p, StaticParams& sp) {
  const double eps = 1e-12;
  auto positive = [&](double v, const char* name) {
    if (!(v > 0))
      return fail(KSIG_ERR_INVALID, "The parameter '%s' should have a positive value.", name);
    return (int)KSIG_OK;
  };
  sp = StaticParams{0.0, 0.0, 0.0};
  int rc = KSIG_OK;
  switch (kind) {
    case KSIG_STATIC_RBF: return positive(p[0], "bandwidth");
    case KSIG_STATIC_LINEAR: return positive(p[0], "scale");
    case KSIG_STATIC_POLY:
      if ((rc = positive(p[0], "degree")) || (rc = positive(p[2], "scale"))) return rc;
      sp = StaticParams{p[1], p[0], p[2]};
      return KSIG_OK;
    case KSIG_STATIC_MATERN12:
    case KSIG_STATIC_MATERN32:
      if ((rc = positive(p[0], "bandwidth"))) return rc;
      sp.c0 = (kind == KSIG_STATIC_MATERN32 ? sqrt(3.0) : 1.0) / fmax(p[0], eps);
      return KSIG_OK;
    case KSIG_STATIC_MATERN52:
      if ((rc = positive(p[0], "bandwidth"))) return rc;
      sp.c0 = 5.0 / fmax(p[0] * p[0], eps);
      return KSIG_OK;
    case KSIG_STATIC_RQ:
      if ((rc = positive(p[0], "bandwidth")) || (rc = positive(p[1], "alpha"))) return rc;
      sp.c0 = 1.0 / fmax(2.0 * p[1] * p[0] * p[0], eps);
      sp.c1 = p[1];
      return KSIG_OK;
  }
  return fail(KSIG_ERR_INVALID, "unknown static kernel %d", kind);
}

int check_common(const void* X, const void* Y, int pairs_mode, const int32_t* list, int n_list,
                 int static_kind, double static_param) {
  if (!X) return fail(KSIG_ERR_INVALID, "X is NULL");
  if ((pairs_mode == KSIG_PAIRS_FULL || pairs_mode == KSIG_PAIRS_LIST) && !Y)
    return fail(KSIG_ERR_INVALID, "Y is NULL");
  if (pairs_mode == KSIG_PAIRS_LIST && (!list || n_list < 0))
    return fail(KSIG_ERR_INVALID, "pair list missing");
  if (static_kind != KSIG_STATIC_RBF && static_kind != KSIG_STATIC_LINEAR)
    return fail(KSIG_ERR_INVALID, "unknown static kernel %d", static_kind);
  if (!(static_param > 0))  // ksig/utils.py:33-34 (check_positive_value)
    return fail(KSIG_ERR_INVALID, "The parameter '%s' should have a positive value.",
                static_kind == KSIG_STATIC_RBF ? "bandwidth" : "scale");
  return KSIG_OK;
}

// The plain one-pair-per-block DP kernel as the generic path for shapes no
// fused instantiation covers (orders above 8, more than 32 levels): any d,
// order and n_levels, same outputs.
int plain_entry(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                const int32_t* lenY, int nY, int LY, int d, int dtype, int static_kind,
                double static_param, int n_levels, int order, int pairs_mode,
                const int32_t* list, int n_list, double* out, void* ws, size_t ws_bytes,
                void* stream) {
  PlainPlan pp;
  int rc = plan_plain(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, pp);
  if (rc) return rc;
  if (!ws || ws_bytes < pp.total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                ws_bytes, pp.total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(ws, 0, 16, st));
  if (pp.f.ntasks == 0) return KSIG_OK;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; Y = X; lenY = lenX; }
  if (dtype == KSIG_DTYPE_F64)
    return run_plain<double>(pp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind, static_param,
                             n_levels, pairs_mode, list, out, static_cast<char*>(ws), st);
  return run_plain<float>(pp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param,
                          n_levels, pairs_mode, list, out, static_cast<char*>(ws), st);
}

int fwd_entry(int family, const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
              const int32_t* lenY, int nY, int LY, int d, int dtype, int static_kind,
              double static_param, int n_levels, int order_or_dyadic, int difference,
              int pairs_mode, const int32_t* list, int n_list, double* out, void* ws,
              size_t ws_bytes, void* stream, bool allow_order = true,
              const double* ext_params = nullptr) {
  // ext_params: the *_ex entry points' parameter list (any static kernel);
  // otherwise RBF / linear with static_param.
  StaticParams sp{0.0, 0.0, 0.0};
  int rc;
  if (ext_params) {
    rc = check_common(X, Y, pairs_mode, list, n_list, KSIG_STATIC_RBF, 1.0);
    if (!rc) rc = static_params(static_kind, ext_params, sp);
    static_param = ext_params[0];
  } else {
    rc = check_common(X, Y, pairs_mode, list, n_list, static_kind, static_param);
  }
  if (rc) return rc;
  if (!out) return fail(KSIG_ERR_INVALID, "output is NULL");
  FwdPlan pl;
  const bool ext = static_kind != KSIG_STATIC_RBF && static_kind != KSIG_STATIC_LINEAR;
  rc = plan_fwd(family, nX, LX, nY, LY, d, dtype, n_levels, order_or_dyadic, difference,
                pairs_mode, n_list, pl, allow_order, ext);
  if (rc == KSIG_ERR_UNSUPPORTED && family == 0 && !ext && difference)
    return plain_entry(X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind, static_param,
                       n_levels, order_or_dyadic, pairs_mode, list, n_list, out, ws, ws_bytes,
                       stream);
  if (rc) return rc;
  if (!ws || ws_bytes < pl.total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                ws_bytes, pl.total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(ws, 0, 16, st));  // device status word
  if (pl.ntasks == 0) return KSIG_OK;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; Y = X; lenY = lenX; }
  const int f64 = dtype == KSIG_DTYPE_F64;
  if (f64)
    return run_fwd<double>(pl, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind, static_param, sp,
                           pairs_mode, list, out, static_cast<char*>(ws), st);
  return run_fwd<float>(pl, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param, sp,
                        pairs_mode, list, out, static_cast<char*>(ws), st);
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void fp32_probe_kernel(float* out, int iters, float a, float b) {
  float v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = threadIdx.x * 1e-3f + i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = fmaf(v[i], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += v[i];
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

// ---- fixed device scratch for ksig_signature_kern_static -----------------
// Some callers of this library cannot allocate device memory: a host that
// binds the C ABI over an FFI and is handed only raw device pointers, a
// framework whose allocator has reserved the device memory up front and
// does not let other code call cudaMalloc, or a latency-bound loop that
// cannot afford the device-wide synchronisation of cudaMalloc / cudaFree.
// For them the forward DP kernel also runs out of this file-scope array.
// Every GPU that loads the library holds it until the process exits, and
// all calls share it.
constexpr size_t kStaticScratchBytes = (size_t)16 << 20;  // 16 MiB
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on the current device.  In host code
// the symbol's name is only a host-side stand-in, never a device address,
// so it is resolved with cudaGetSymbolAddress, with the device current.  It
// is looked up on every call (cheap once the module is loaded), so the
// address stays right after a cudaDeviceReset reloads the module; the first
// lookup on a device loads the module, which is why the first call of
// ksig_signature_kern_static on a device should come before any stream
// capture.
void* static_scratch_ptr(cudaError_t* err) {
  void* p = nullptr;
  *err = cudaGetSymbolAddress(&p, g_static_scratch);
  return *err == cudaSuccess ? p : nullptr;
}

}  // namespace
}  // namespace ksig

using namespace ksig;

extern "C" {

const char* ksig_version(void) { return "ksig_b200 0.1.0 (sm_100a)"; }

size_t ksig_last_error(char* buf, size_t n) {
  if (buf && n) {
    size_t m = g_err.size() < n - 1 ? g_err.size() : n - 1;
    memcpy(buf, g_err.data(), m);
    buf[m] = 0;
  }
  return g_err.size();
}

long long ksig_num_pairs(int pairs_mode, int nX, int nY, int n_list) {
  return num_pairs(pairs_mode, nX, nY, n_list);
}

size_t ksig_signature_kern_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                     int n_levels, int order, int difference, int pairs_mode,
                                     int n_list) {
  FwdPlan pl;
  if (int rc = plan_fwd(false, nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode,
                        n_list, pl)) {
    // No fused instantiation: the plain kernel's workspace (fwd_entry).
    PlainPlan pp;
    if (rc == KSIG_ERR_UNSUPPORTED && difference &&
        !plan_plain(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, pp))
      return pp.total;
    return 0;
  }
  // Also large enough for the other static kernels' instantiations
  // (ksig_signature_kern_ex), where one is compiled for this shape.
  FwdPlan px;
  if (!plan_fwd(false, nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode, n_list,
                px, true, true) &&
      px.total > pl.total)
    return px.total;
  return pl.total;
}

int ksig_signature_kern(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                        const int32_t* lenY, int nY, int LY, int d, int dtype, int static_kind,
                        double static_param, int n_levels, int order, int difference,
                        int pairs_mode, const int32_t* pair_list, int n_list, double* out_levels,
                        void* workspace, size_t workspace_bytes, void* stream) {
  return fwd_entry(false, X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind, static_param,
                   n_levels, order, difference, pairs_mode, pair_list, n_list, out_levels,
                   workspace, workspace_bytes, stream);
}

size_t ksig_signature_kern_pde_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                         int dyadic_order, int difference, int pairs_mode,
                                         int n_list) {
  FwdPlan pl;
  if (plan_fwd(true, nX, LX, nY, LY, d, dtype, 0, dyadic_order, difference, pairs_mode, n_list,
               pl))
    return 0;
  FwdPlan px;
  if (!plan_fwd(true, nX, LX, nY, LY, d, dtype, 0, dyadic_order, difference, pairs_mode, n_list,
                px, true, true) &&
      px.total > pl.total)
    return px.total;
  return pl.total;
}

int ksig_signature_kern_pde(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                            const int32_t* lenY, int nY, int LY, int d, int dtype,
                            int static_kind, double static_param, int dyadic_order,
                            int difference, int pairs_mode, const int32_t* pair_list, int n_list,
                            double* out, void* workspace, size_t workspace_bytes, void* stream) {
  return fwd_entry(true, X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind, static_param,
                   0, dyadic_order, difference, pairs_mode, pair_list, n_list, out, workspace,
                   workspace_bytes, stream);
}

int ksig_signature_kern_ex(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                           const int32_t* lenY, int nY, int LY, int d, int dtype,
                           int static_kind, const double* static_params, int n_levels, int order,
                           int difference, int pairs_mode, const int32_t* pair_list, int n_list,
                           double* out_levels, void* workspace, size_t workspace_bytes,
                           void* stream) {
  if (!static_params) return fail(KSIG_ERR_INVALID, "static_params is NULL");
  return fwd_entry(false, X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind,
                   static_params[0], n_levels, order, difference, pairs_mode, pair_list, n_list,
                   out_levels, workspace, workspace_bytes, stream, true, static_params);
}

int ksig_signature_kern_pde_ex(const void* X, const int32_t* lenX, int nX, int LX,
                               const void* Y, const int32_t* lenY, int nY, int LY, int d,
                               int dtype, int static_kind, const double* static_params,
                               int dyadic_order, int difference, int pairs_mode,
                               const int32_t* pair_list, int n_list, double* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (!static_params) return fail(KSIG_ERR_INVALID, "static_params is NULL");
  return fwd_entry(true, X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind,
                   static_params[0], 0, dyadic_order, difference, pairs_mode, pair_list, n_list,
                   out, workspace, workspace_bytes, stream, true, static_params);
}

size_t ksig_global_align_kern_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                        int pairs_mode, int n_list) {
  FwdPlan pl;
  if (plan_fwd(2, nX, LX, nY, LY, d, dtype, 0, 0, 0, pairs_mode, n_list, pl)) return 0;
  return pl.total;
}

int ksig_global_align_kern(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                           const int32_t* lenY, int nY, int LY, int d, int dtype,
                           int static_kind, double static_param, int pairs_mode,
                           const int32_t* pair_list, int n_list, double* out_log,
                           void* workspace, size_t workspace_bytes, void* stream) {
  return fwd_entry(2, X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind, static_param, 0,
                   0, 0, pairs_mode, pair_list, n_list, out_log, workspace, workspace_bytes,
                   stream);
}

int ksig_signature_kern_static(const void* X, const int32_t* lenX, int nX, int LX,
                               const void* Y, const int32_t* lenY, int nY, int LY, int d,
                               int dtype, int static_kind, double static_param, int n_levels,
                               int order, int difference, int pairs_mode,
                               const int32_t* pair_list, int n_list, double* out_levels,
                               void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  // The fixed scratch holds no task-order buffers: tasks run in natural order.
  FwdPlan pl;
  rc = plan_fwd(false, nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode,
                n_list, pl, false);
  if (rc) return rc;
  if (pl.total > kStaticScratchBytes)
    return fail(KSIG_ERR_WORKSPACE,
                "this call needs %zu bytes of scratch, more than the %zu-byte static scratch "
                "of ksig_signature_kern_static; call ksig_signature_kern with a workspace",
                pl.total, kStaticScratchBytes);
  cudaError_t e = cudaSuccess;
  void* ws = static_scratch_ptr(&e);
  if (!ws) return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
  return fwd_entry(false, X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind, static_param,
                   n_levels, order, difference, pairs_mode, pair_list, n_list, out_levels, ws,
                   kStaticScratchBytes, stream, false);
}

size_t ksig_signature_kern_plain_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                           int n_levels, int order, int pairs_mode, int n_list) {
  PlainPlan pp;
  if (plan_plain(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, pp)) return 0;
  return pp.total;
}

int ksig_signature_kern_plain(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                              const int32_t* lenY, int nY, int LY, int d, int dtype,
                              int static_kind, double static_param, int n_levels, int order,
                              int pairs_mode, const int32_t* pair_list, int n_list,
                              double* out_levels, void* workspace, size_t workspace_bytes,
                              void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  if (!out_levels) return fail(KSIG_ERR_INVALID, "output is NULL");
  PlainPlan pp;
  rc = plan_plain(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, pp);
  if (rc) return rc;
  if (!workspace || workspace_bytes < pp.total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                workspace_bytes, pp.total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
  if (pp.f.ntasks == 0) return KSIG_OK;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; Y = X; lenY = lenX; }
  if (dtype == KSIG_DTYPE_F64)
    return run_plain<double>(pp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind,
                             static_param, n_levels, pairs_mode, pair_list, out_levels,
                             static_cast<char*>(workspace), st);
  return run_plain<float>(pp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param,
                          n_levels, pairs_mode, pair_list, out_levels,
                          static_cast<char*>(workspace), st);
}

size_t ksig_signature_kern_plain_bwd_workspace(int nX, int LX, int nY, int LY, int d,
                                               int dtype, int n_levels, int order,
                                               int pairs_mode, int n_list) {
  PlainBwdPlan bp;
  if (plan_plain_bwd(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, bp))
    return 0;
  return bp.pp.total;
}

int ksig_signature_kern_plain_bwd(const void* X, const int32_t* lenX, int nX, int LX,
                                  const void* Y, const int32_t* lenY, int nY, int LY, int d,
                                  int dtype, int static_kind, double static_param, int n_levels,
                                  int order, int pairs_mode, const int32_t* pair_list,
                                  int n_list, const double* grad_levels, void* dX,
                                  double* dparam, void* workspace, size_t workspace_bytes,
                                  void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  if (!grad_levels || !dX) return fail(KSIG_ERR_INVALID, "grad_levels or dX is NULL");
  PlainBwdPlan bp;
  rc = plan_plain_bwd(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, bp);
  if (rc) return rc;
  if (!workspace || workspace_bytes < bp.pp.total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                workspace_bytes, bp.pp.total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
  if (bp.pp.f.ntasks == 0) return KSIG_OK;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; Y = X; lenY = lenX; }
  const int nl_out = n_levels;
  if (dtype == KSIG_DTYPE_F64)
    return run_plain_bwd<double>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind,
                                 static_param, n_levels, pairs_mode, pair_list, grad_levels,
                                 nl_out, dX, dparam, static_cast<char*>(workspace), st);
  return run_plain_bwd<float>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind,
                              static_param, n_levels, pairs_mode, pair_list, grad_levels, nl_out,
                              dX, dparam, static_cast<char*>(workspace), st);
}

size_t ksig_signature_kern_bwd_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                         int n_levels, int order, int difference,
                                         int pairs_mode, int n_list) {
  BwdPlan bp;
  if (int rc = plan_bwd(nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode,
                        n_list, bp)) {
    // No fused adjoint for this shape: the plain adjoint's workspace.
    PlainBwdPlan pb;
    if (rc == KSIG_ERR_UNSUPPORTED && difference &&
        !plan_plain_bwd(nX, LX, nY, LY, d, dtype, n_levels, order, pairs_mode, n_list, pb))
      return pb.pp.total;
    return 0;
  }
  return bp.total;
}

int ksig_signature_kern_bwd(const void* X, const int32_t* lenX, int nX, int LX, const void* Y,
                            const int32_t* lenY, int nY, int LY, int d, int dtype,
                            int static_kind, double static_param, int n_levels, int order,
                            int difference, int pairs_mode, const int32_t* pair_list, int n_list,
                            const double* grad_levels, void* dX, double* dparam,
                            void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  if (!grad_levels || !dX) return fail(KSIG_ERR_INVALID, "grad_levels / dX is NULL");
  BwdPlan bp;
  rc = plan_bwd(nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode, n_list, bp);
  if (rc == KSIG_ERR_UNSUPPORTED && difference)
    // Shapes no fused adjoint covers (d above 32, orders above 8, more than
    // 32 levels): the plain one-pair-per-block adjoint, same results.
    return ksig_signature_kern_plain_bwd(X, lenX, nX, LX, Y, lenY, nY, LY, d, dtype, static_kind,
                                         static_param, n_levels, order, pairs_mode, pair_list,
                                         n_list, grad_levels, dX, dparam, workspace,
                                         workspace_bytes, stream);
  if (rc) return rc;
  if (!workspace || workspace_bytes < bp.total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                workspace_bytes, bp.total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
  if (bp.f.ntasks == 0) return KSIG_OK;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; Y = X; lenY = lenX; }
  if (dtype == KSIG_DTYPE_F64)
    return run_bwd<double>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind, static_param,
                           pairs_mode, pair_list, grad_levels, n_levels, dX, dparam,
                           static_cast<char*>(workspace), st);
  return run_bwd<float>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param,
                        pairs_mode, pair_list, grad_levels, n_levels, dX, dparam,
                        static_cast<char*>(workspace), st);
}

// Split gradient pass (order 1): the forward pass of the adjoint kernel
// with its per-pair records kept in the workspace, then the adjoint pass
// replaying them.  One plan serves both calls.
static int rec_plan(int nX, int LX, int nY, int LY, int d, int dtype, int n_levels, int order,
                    int difference, int pairs_mode, int n_list, BwdPlan& bp, size_t& total) {
  if (pairs_mode != KSIG_PAIRS_FULL && pairs_mode != KSIG_PAIRS_LIST)
    return fail(KSIG_ERR_UNSUPPORTED, "the split gradient pass takes full or listed pairs");
  int rc = plan_bwd(nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode, n_list, bp,
                    false);
  if (rc) return rc;
  if (bp.f.p != 1 || n_levels < 2)
    return fail(KSIG_ERR_UNSUPPORTED, "the split gradient pass needs order 1 and n_levels >= 2");
  if (!rec_fwd_entry(bp))
    return fail(KSIG_ERR_UNSUPPORTED, "no compiled split forward pass for this tile");
  const size_t es = bp.f.f64 ? 8 : 4;
  total = align_up(bp.total + (size_t)bp.f.ntasks * (size_t)bp.rec_per_pair * es);
  return KSIG_OK;
}

size_t ksig_signature_kern_rec_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                         int n_levels, int order, int difference,
                                         int pairs_mode, int n_list) {
  BwdPlan bp;
  size_t total = 0;
  if (rec_plan(nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode, n_list, bp,
               total))
    return 0;
  return total;
}

int ksig_signature_kern_rec_fwd(const void* X, const int32_t* lenX, int nX, int LX,
                                const void* Y, const int32_t* lenY, int nY, int LY, int d,
                                int dtype, int static_kind, double static_param, int n_levels,
                                int order, int difference, int pairs_mode,
                                const int32_t* pair_list, int n_list, double* levels,
                                void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  if (!levels) return fail(KSIG_ERR_INVALID, "levels is NULL");
  BwdPlan bp;
  size_t total = 0;
  rc = rec_plan(nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode, n_list, bp,
                total);
  if (rc) return rc;
  if (!workspace || workspace_bytes < total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                workspace_bytes, total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
  KSIG_CUDA(cudaMemsetAsync(levels, 0, sizeof(double) * (size_t)(n_levels + 1) * bp.f.ntasks, st));
  if (bp.f.ntasks == 0) return KSIG_OK;
  char* ws = static_cast<char*>(workspace);
  if (dtype == KSIG_DTYPE_F64)
    return run_bwd<double>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind, static_param,
                           pairs_mode, pair_list, nullptr, n_levels, nullptr, nullptr, ws, st, 1,
                           levels);
  return run_bwd<float>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param,
                        pairs_mode, pair_list, nullptr, n_levels, nullptr, nullptr, ws, st, 1,
                        levels);
}

int ksig_signature_kern_rec_bwd(const void* X, const int32_t* lenX, int nX, int LX,
                                const void* Y, const int32_t* lenY, int nY, int LY, int d,
                                int dtype, int static_kind, double static_param, int n_levels,
                                int order, int difference, int pairs_mode,
                                const int32_t* pair_list, int n_list, const double* grad_levels,
                                void* dX, double* dparam, void* workspace,
                                size_t workspace_bytes, void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  if (!grad_levels || !dX) return fail(KSIG_ERR_INVALID, "grad_levels / dX is NULL");
  BwdPlan bp;
  size_t total = 0;
  rc = rec_plan(nX, LX, nY, LY, d, dtype, n_levels, order, difference, pairs_mode, n_list, bp,
                total);
  if (rc) return rc;
  if (!workspace || workspace_bytes < total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                workspace_bytes, total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
  if (bp.f.ntasks == 0) return KSIG_OK;
  char* ws = static_cast<char*>(workspace);
  if (dtype == KSIG_DTYPE_F64)
    return run_bwd<double>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind, static_param,
                           pairs_mode, pair_list, grad_levels, n_levels, dX, dparam, ws, st, 2);
  return run_bwd<float>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param,
                        pairs_mode, pair_list, grad_levels, n_levels, dX, dparam, ws, st, 2);
}

size_t ksig_signature_kern_pde_bwd_workspace(int nX, int LX, int nY, int LY, int d, int dtype,
                                             int dyadic_order, int difference, int pairs_mode,
                                             int n_list) {
  PdeBwdPlan bp;
  if (plan_pde_bwd(nX, LX, nY, LY, d, dtype, dyadic_order, difference, pairs_mode, n_list, bp))
    return 0;
  return bp.total;
}

int ksig_signature_kern_pde_bwd(const void* X, const int32_t* lenX, int nX, int LX,
                                const void* Y, const int32_t* lenY, int nY, int LY, int d,
                                int dtype, int static_kind, double static_param,
                                int dyadic_order, int difference, int pairs_mode,
                                const int32_t* pair_list, int n_list, const double* grad,
                                void* dX, double* dparam, void* workspace,
                                size_t workspace_bytes, void* stream) {
  int rc = check_common(X, Y, pairs_mode, pair_list, n_list, static_kind, static_param);
  if (rc) return rc;
  if (!grad || !dX) return fail(KSIG_ERR_INVALID, "grad / dX is NULL");
  PdeBwdPlan bp;
  rc = plan_pde_bwd(nX, LX, nY, LY, d, dtype, dyadic_order, difference, pairs_mode, n_list, bp);
  if (rc) return rc;
  if (!workspace || workspace_bytes < bp.total)
    return fail(KSIG_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                workspace_bytes, bp.total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KSIG_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
  if (bp.f.ntasks == 0) return KSIG_OK;
  if (pairs_mode == KSIG_PAIRS_UPPER || pairs_mode == KSIG_PAIRS_DIAG) { nY = nX; LY = LX; Y = X; lenY = lenX; }
  if (dtype == KSIG_DTYPE_F64)
    return run_pde_bwd<double>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 1, static_kind,
                               static_param, pairs_mode, pair_list, grad, dX, dparam,
                               static_cast<char*>(workspace), st);
  return run_pde_bwd<float>(bp, X, lenX, nX, LX, Y, lenY, nY, LY, d, 0, static_kind, static_param,
                            pairs_mode, pair_list, grad, dX, dparam,
                            static_cast<char*>(workspace), st);
}

int ksig_normalize_levels(const double* levels, int n_lev, int pairs_mode, int nX, int nY,
                          const double* diagX, const double* diagY, int normalize, void* out,
                          int out_dtype, void* stream) {
  if (!levels || !out) return fail(KSIG_ERR_INVALID, "NULL levels/out");
  if (n_lev <= 0 || nX <= 0) return fail(KSIG_ERR_INVALID, "bad sizes");
  if (pairs_mode != KSIG_PAIRS_FULL && pairs_mode != KSIG_PAIRS_UPPER)
    return fail(KSIG_ERR_INVALID, "normalize needs FULL or UPPER pairs");
  if (pairs_mode == KSIG_PAIRS_UPPER) nY = nX;
  if (nY <= 0) return fail(KSIG_ERR_INVALID, "bad nY");
  if (normalize && !diagX && pairs_mode == KSIG_PAIRS_FULL && nX != nY)
    return fail(KSIG_ERR_INVALID, "diagX is required for a rectangular FULL Gram");
  if (out_dtype != KSIG_DTYPE_F32 && out_dtype != KSIG_DTYPE_F64)
    return fail(KSIG_ERR_INVALID, "bad out dtype");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  NormArgs a{levels, n_lev, pairs_mode, nX, nY, diagX, diagY ? diagY : diagX, normalize};
  const long long total = (long long)nX * nY;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 8192) blocks = 8192;
  if (out_dtype == KSIG_DTYPE_F64) normalize_kernel<double><<<blocks, 256, 0, st>>>(a, (double*)out);
  else normalize_kernel<float><<<blocks, 256, 0, st>>>(a, (float*)out);
  KSIG_CUDA(cudaGetLastError());
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return KSIG_OK;
}

unsigned long long ksig_launch_count(void) { return g_launches.load(); }

void ksig_profile_enable(int on) {
  Profiler& P = prof();
  std::lock_guard<std::mutex> lk(P.mu);
  P.on = on != 0;
}

int ksig_profile_read(double* total_ms, long long* launches) {
  Profiler& P = prof();
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  {
    std::lock_guard<std::mutex> lk(P.mu);
    ev.swap(P.pending);
  }
  double tot = 0.0;
  for (auto& e : ev) {
    KSIG_CUDA(cudaEventSynchronize(e.second));
    float ms = 0.f;
    KSIG_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
    tot += ms;
  }
  {
    std::lock_guard<std::mutex> lk(P.mu);
    for (auto& e : ev) P.pool.push_back(e);
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = (long long)ev.size();
  return KSIG_OK;
}

int ksig_tune_set_cols(int op, int cols) {
  if (op < 0 || op > 3) return fail(KSIG_ERR_INVALID, "bad kernel family %d", op);
  if (cols < 0 || cols > 32) return fail(KSIG_ERR_INVALID, "bad column count %d", cols);
  g_tuned_cols[op].store(cols);
  return KSIG_OK;
}

int ksig_tune_get_cols(int op) { return tuned_cols(op); }

int ksig_fp32_peak(double* tflops, void* stream) {
  if (!tflops) return fail(KSIG_ERR_INVALID, "NULL output");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int sms = sm_count() > 0 ? sm_count() : 148;
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t a, b;
  KSIG_CUDA(cudaEventCreate(&a));
  KSIG_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    KSIG_CUDA(cudaEventRecord(a, st));
    fp32_probe_kernel<<<blocks, threads, 0, st>>>(nullptr, iters, 0.999f, 1e-3f);
    KSIG_CUDA(cudaGetLastError());
    KSIG_CUDA(cudaEventRecord(b, st));
    KSIG_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    KSIG_CUDA(cudaEventElapsedTime(&ms, a, b));
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return KSIG_OK;
}

int ksig_static_status(void* stream) {
  cudaError_t e = cudaSuccess;
  void* ws = static_scratch_ptr(&e);
  if (!ws) return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
  return ksig_workspace_status(ws, stream);
}

int ksig_workspace_status(void* workspace, void* stream) {
  if (!workspace) return fail(KSIG_ERR_INVALID, "NULL workspace");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int h = 0;
  KSIG_CUDA(cudaMemcpyAsync(&h, workspace, sizeof(int), cudaMemcpyDeviceToHost, st));
  KSIG_CUDA(cudaStreamSynchronize(st));
  if (h != 0) {
    int z = 0;
    KSIG_CUDA(cudaMemcpyAsync(workspace, &z, sizeof(int), cudaMemcpyHostToDevice, st));
    KSIG_CUDA(cudaStreamSynchronize(st));
    return fail(h == KSIG_ERR_INVALID ? KSIG_ERR_INVALID : KSIG_ERR_DEVICE,
                "device-side check failed (code %d)", h);
  }
  return KSIG_OK;
}

}  // extern "C"
