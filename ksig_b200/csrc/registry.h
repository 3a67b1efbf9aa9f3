// Table of compiled kernel instantiations, filled by the generated
// translation units under csrc/gen/ (see build.py for the instance list).
#pragma once

#include <cuda_runtime.h>

namespace ksig {

enum KernelOp : int {
  OP_DP_FWD = 0,   // SweepArgs<T>          dp_fwd_kernel
  OP_PDE_FWD = 1,  // SweepArgs<T>          pde_fwd_kernel   (p = refinement F)
  OP_DP_BWD = 2,   // DpBwdArgs<T>          dp_bwd_kernel
  OP_PDE_BWD = 3,  // PdeBwdArgs<T>         pde_bwd_kernel
  OP_DP_FWD_EXT = 4,   // dp_fwd_kernel, EXT: the other static kernels
  OP_PDE_FWD_EXT = 5,  // pde_fwd_kernel, EXT
  OP_GA_FWD = 6,       // SweepArgs<T>      ga_fwd_kernel (global alignment)
  OP_DP_REC_FWD = 7,   // DpBwdArgs<T>      dp_rec_fwd_kernel (split gradient pass)
  OP_DP_BWD_CKPT = 8,  // DpBwdArgs<T>      dp_bwd_ckpt_kernel (strip checkpointing)
  OP_PDE_FWD_STACK = 9,  // SweepArgs<T>    pde_fwd_kernel, stacked pairs (STK)
};

struct KernelEntry {
  int op, f64, kd, c, nl, p, diff, wpb;
  const void* func;
};

struct KernelTable {
  const KernelEntry* entries;
  int n;
};

// All tables (defined in the generated registry translation unit).
extern const KernelTable kAllTables[];
extern const int kNumTables;

}  // namespace ksig
