/*
 * ksig_b200 — C ABI of the B200 (sm_100a) signature-kernel library.
 *
 * Every entry point takes caller-owned DEVICE pointers, a caller-owned
 * device workspace, and a cudaStream_t passed as `void*` (NULL = legacy
 * default stream).  Calls are asynchronous on that stream except where a
 * function says otherwise; they return a KSIG_* status code and never
 * allocate device memory.  Sequences are dense row-major arrays
 * [n, L, d] of float32 or float64 (dtype KSIG_DTYPE_*); an optional int32
 * device array `len[n]` gives each sequence's true number of points
 * (2..L; points past it are ignored, which is exactly the reference's
 * behaviour on edge-padded arrays).  The arithmetic runs in the input
 * dtype (float32 inputs: FP32 with FP64 level/normalisation reductions;
 * float64 inputs: FP64 throughout).
 *
 * Reference interfaces replaced (tgcsaba/KSig 1.0.0, paths within the
 * project):
 *   ksig_signature_kern      SignatureKernel._compute_kernel
 *                            (ksig/kernels.py:147-164) = _compute_embedding
 *                            (ksig/kernels.py:124-145, static Gram through
 *                            RBFKernel._K ksig/static/kernels.py:248-260 or
 *                            LinearKernel._K :145-155) followed by
 *                            signature_kern(..., return_levels=True)
 *                            (ksig/algorithms.py:22-140).
 *   ksig_signature_kern_pde  SignaturePDEKernel._compute_kernel
 *                            (ksig/kernels.py:242-256) = static Gram +
 *                            signature_kern_pde (ksig/algorithms.py:402-446)
 *                            and its Numba kernel (:344-399).
 *   ksig_normalize_levels    the normalisation and level mean of
 *                            SignatureKernel._K (ksig/kernels.py:190-214),
 *                            robust_sqrt (ksig/utils.py:173-182).
 *   ksig_*_bwd               no reference counterpart (the reference has no
 *                            gradients); adjoints of the two kernels above.
 */
#ifndef KSIG_B200_H_
#define KSIG_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define KSIG_OK 0
#define KSIG_ERR_INVALID 1     /* invalid argument (shape, parameter, dtype) */
#define KSIG_ERR_UNSUPPORTED 2 /* no compiled kernel for this configuration  */
#define KSIG_ERR_WORKSPACE 3   /* workspace smaller than required            */
#define KSIG_ERR_CUDA 4        /* CUDA runtime error (see ksig_last_error)   */
#define KSIG_ERR_DEVICE 5      /* device-side check failed (bounded wait,
                                  bounds check); the context stays usable    */

/* Static (state-space) kernels.  The *_ex entry points take the parameter
 * list shown in braces (ksig/static/kernels.py:137-343); the others take
 * the one parameter of RBF and linear. */
#define KSIG_STATIC_RBF 0       /* {s}: exp(-|x-y|^2 / max(2 s^2, 1e-12))        */
#define KSIG_STATIC_LINEAR 1    /* {s}: s <x, y>                                  */
#define KSIG_STATIC_POLY 2      /* {degree, gamma, scale}:
                                   scale (<x, y> + gamma)^degree                 */
#define KSIG_STATIC_MATERN12 3  /* {s}: exp(-D), D = |x-y| / s                   */
#define KSIG_STATIC_MATERN32 4  /* {s}: (1 + D) exp(-D), D = sqrt(3) |x-y| / s   */
#define KSIG_STATIC_MATERN52 5  /* {s}: (1 + D + D^2/3) exp(-D), D = sqrt(5) |x-y| / s */
#define KSIG_STATIC_RQ 6        /* {s, a}: (1 + |x-y|^2 / (2 a s^2))^-a           */

/* Element types. */
#define KSIG_DTYPE_F32 0
#define KSIG_DTYPE_F64 1

/* Which (row, column) sequence pairs a call evaluates; output entry p of a
 * per-pair array belongs to pair p of this enumeration. */
#define KSIG_PAIRS_FULL 0  /* all nX*nY pairs, p = a*nY + b                  */
#define KSIG_PAIRS_UPPER 1 /* X against itself, a <= b, row-major triangle;
                              p = a*nX - a*(a-1)/2 + (b-a); Y is ignored      */
#define KSIG_PAIRS_DIAG 2  /* (a, a) for a < nX; Y is ignored                 */
#define KSIG_PAIRS_LIST 3  /* explicit int32 pairs (a, b), pair_list[2p..2p+1]*/

/* Library version string. */
const char* ksig_version(void);

/* Copies the message of the last failing call on this host thread into buf
 * (NUL-terminated, truncated to n bytes); returns its full length. */
size_t ksig_last_error(char* buf, size_t n);

/* Number of pairs a pairs_mode enumerates. */
long long ksig_num_pairs(int pairs_mode, int nX, int nY, int n_list);

/* Workspace (bytes) required by ksig_signature_kern with these sizes. */
size_t ksig_signature_kern_workspace(int nX, int LX, int nY, int LY, int d,
                                     int dtype, int n_levels, int order,
                                     int difference, int pairs_mode,
                                     int n_list);

/*
 * Truncated signature kernel per level (replaces
 * SignatureKernel._compute_kernel with return_levels=True,
 * ksig/kernels.py:147-164 and ksig/algorithms.py:22-140).
 *
 *   out_levels  float64 [n_levels + 1, P] with P = ksig_num_pairs(...);
 *               row 0 is 1 (level 0), row k the level-k kernel.
 *   order       Alg. 3 when the clamped order is 1, Alg. 6 otherwise; the
 *               clamp is that of ksig/algorithms.py:37 (order <= 0 or
 *               order >= n_levels -> n_levels).
 *   difference  1: increments of the lifted paths (second difference of the
 *               static Gram, ksig/algorithms.py:63-64); 0: the Gram itself.
 */
int ksig_signature_kern(const void* X, const int32_t* lenX, int nX, int LX,
                        const void* Y, const int32_t* lenY, int nY, int LY,
                        int d, int dtype, int static_kind,
                        double static_param, int n_levels, int order,
                        int difference, int pairs_mode,
                        const int32_t* pair_list, int n_list,
                        double* out_levels, void* workspace,
                        size_t workspace_bytes, void* stream);

/*
 * ksig_signature_kern without a caller workspace.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory (an
 * FFI host holding only raw device pointers, a framework whose allocator
 * owns the device memory, a loop that cannot take cudaMalloc's device-wide
 * synchronisation).  Its scratch is a 16 MiB array compiled into the
 * library: every GPU that loads the library holds it until the process
 * exits.  Tasks run in their natural order (no longest-first order buffers),
 * so a call needs the workspace of that unordered plan, which is at most
 * ksig_signature_kern_workspace(...); calls whose unordered plan exceeds
 * 16 MiB are rejected with KSIG_ERR_WORKSPACE.  It calls no cudaMalloc /
 * cudaFree.  Every call looks up the array's device address
 * (cudaGetSymbolAddress) with the call's device current; the first lookup
 * on a device loads the library's device code there, so make the first call
 * on each device before any stream capture.  All calls share the array and
 * keep the last call's contents (each call clears what must start at zero),
 * so calls that overlap on the GPU race: order them on one stream or
 * synchronise.  Lengths outside [1, L] are clamped and flagged in the
 * array's status word; ksig_static_status reads it.
 */
int ksig_signature_kern_static(const void* X, const int32_t* lenX, int nX,
                               int LX, const void* Y, const int32_t* lenY,
                               int nY, int LY, int d, int dtype,
                               int static_kind, double static_param,
                               int n_levels, int order, int difference,
                               int pairs_mode, const int32_t* pair_list,
                               int n_list, double* out_levels, void* stream);

/*
 * Plain FP32 one-pair-per-block form of ksig_signature_kern (difference=1):
 * the measurement baseline the fused sweep is compared with.  No reference
 * counterpart as an entry point: it evaluates the reference's recursion
 * (ksig/algorithms.py:47-140) as a direct CUDA translation, one CTA per
 * pair with Z and the level states materialised in workspace scratch.
 * Same arguments and output as ksig_signature_kern; order <= 4.
 */
size_t ksig_signature_kern_plain_workspace(int nX, int LX, int nY, int LY,
                                           int d, int dtype, int n_levels,
                                           int order, int pairs_mode,
                                           int n_list);
int ksig_signature_kern_plain(const void* X, const int32_t* lenX, int nX,
                              int LX, const void* Y, const int32_t* lenY,
                              int nY, int LY, int d, int dtype,
                              int static_kind, double static_param,
                              int n_levels, int order, int pairs_mode,
                              const int32_t* pair_list, int n_list,
                              double* out_levels, void* workspace,
                              size_t workspace_bytes, void* stream);

/*
 * Plain FP32 one-pair-per-block form of ksig_signature_kern_bwd
 * (difference=1): the baseline of the fused adjoint.  No reference
 * counterpart (the reference has no gradients).  One CTA per pair keeps Z,
 * every level's states and the adjoint states as full arrays in workspace
 * scratch and runs the adjoint recursion as array passes.  Same arguments
 * and accumulation semantics as ksig_signature_kern_bwd without
 * `difference`; order <= 4.
 */
size_t ksig_signature_kern_plain_bwd_workspace(int nX, int LX, int nY, int LY,
                                               int d, int dtype, int n_levels,
                                               int order, int pairs_mode,
                                               int n_list);
int ksig_signature_kern_plain_bwd(const void* X, const int32_t* lenX, int nX,
                                  int LX, const void* Y, const int32_t* lenY,
                                  int nY, int LY, int d, int dtype,
                                  int static_kind, double static_param,
                                  int n_levels, int order, int pairs_mode,
                                  const int32_t* pair_list, int n_list,
                                  const double* grad_levels, void* dX,
                                  double* dparam, void* workspace,
                                  size_t workspace_bytes, void* stream);

/* Workspace (bytes) required by ksig_signature_kern_pde. */
size_t ksig_signature_kern_pde_workspace(int nX, int LX, int nY, int LY,
                                         int d, int dtype, int dyadic_order,
                                         int difference, int pairs_mode,
                                         int n_list);

/*
 * Signature-PDE kernel (replaces SignaturePDEKernel._compute_kernel,
 * ksig/kernels.py:242-256, and signature_kern_pde,
 * ksig/algorithms.py:402-446).  Second-order Goursat scheme of
 * ksig/algorithms.py:384-385 with boundary value 1.  dyadic_order k > 0
 * refines every cell into 2^k x 2^k cells with increment q / 4^k (no
 * reference counterpart; k = 0 is the reference scheme).
 *   out  float64 [P].
 */
int ksig_signature_kern_pde(const void* X, const int32_t* lenX, int nX,
                            int LX, const void* Y, const int32_t* lenY,
                            int nY, int LY, int d, int dtype,
                            int static_kind, double static_param,
                            int dyadic_order, int difference, int pairs_mode,
                            const int32_t* pair_list, int n_list,
                            double* out, void* workspace,
                            size_t workspace_bytes, void* stream);

/*
 * ksig_signature_kern and ksig_signature_kern_pde for every static kernel
 * of ksig.static.kernels: `static_params` holds the kind's parameters as
 * listed with KSIG_STATIC_* (up to 3 values; positive where the reference
 * requires it, ksig/utils.py:23-35).  Same workspace as the plain entry
 * points.  The adjoint entry points support RBF and linear only.
 */
int ksig_signature_kern_ex(const void* X, const int32_t* lenX, int nX, int LX,
                           const void* Y, const int32_t* lenY, int nY, int LY,
                           int d, int dtype, int static_kind,
                           const double* static_params, int n_levels,
                           int order, int difference, int pairs_mode,
                           const int32_t* pair_list, int n_list,
                           double* out_levels, void* workspace,
                           size_t workspace_bytes, void* stream);
int ksig_signature_kern_pde_ex(const void* X, const int32_t* lenX, int nX,
                               int LX, const void* Y, const int32_t* lenY,
                               int nY, int LY, int d, int dtype,
                               int static_kind, const double* static_params,
                               int dyadic_order, int difference,
                               int pairs_mode, const int32_t* pair_list,
                               int n_list, double* out, void* workspace,
                               size_t workspace_bytes, void* stream);

/* Workspace (bytes) required by ksig_global_align_kern. */
size_t ksig_global_align_kern_workspace(int nX, int LX, int nY, int LY, int d,
                                        int dtype, int pairs_mode, int n_list);

/*
 * Global alignment kernel in log space (replaces global_align_kern_log,
 * ksig/algorithms.py:453-559, behind GlobalAlignmentKernel._compute_kernel,
 * ksig/kernels.py:366-409).  With M the static Gram of the pair (RBF or
 * linear, no differencing), M' = M / (2 - M), logM = log(max(M', 1e-12)):
 *   logK[i,j] = logM[i,j] + logsumexp(logK[i-1,j], logK[i,j-1], logK[i-1,j-1]),
 * logK[-1,-1] = 0, -inf elsewhere on the boundary.
 *   out_log  float64 [P]: logK at the last point pair of every pair.
 * The normalisation of GlobalAlignmentKernel (log-space, ksig/kernels.py:
 * 190-206) is left to the caller.
 */
int ksig_global_align_kern(const void* X, const int32_t* lenX, int nX,
                           int LX, const void* Y, const int32_t* lenY, int nY,
                           int LY, int d, int dtype, int static_kind,
                           double static_param, int pairs_mode,
                           const int32_t* pair_list, int n_list,
                           double* out_log, void* workspace,
                           size_t workspace_bytes, void* stream);

/* Workspace (bytes) required by ksig_signature_kern_bwd. */
size_t ksig_signature_kern_bwd_workspace(int nX, int LX, int nY, int LY,
                                         int d, int dtype, int n_levels,
                                         int order, int difference,
                                         int pairs_mode, int n_list);

/*
 * Adjoint of ksig_signature_kern (no reference counterpart: the reference
 * has no gradients).  For every pair p = (a, b) of the enumeration and
 * grad_levels[k, p] = dL/dlevel_k(p) (float64 [n_levels + 1, P], row 0
 * ignored) it accumulates
 *   dX[a]   += sum_k grad_levels[k, p] * d level_k(x_a, y_b) / d x_a
 *   *dparam += sum_k grad_levels[k, p] * d level_k(x_a, y_b) / d param
 * dX has X's dtype and shape [nX, LX, d] and is NOT cleared; only the ROW
 * sequence of each pair is differentiated (call again with the roles
 * swapped for the column side).  dparam (float64 scalar, may be NULL) is the
 * RBF bandwidth or the linear scale.  difference must be 1.
 */
int ksig_signature_kern_bwd(const void* X, const int32_t* lenX, int nX,
                            int LX, const void* Y, const int32_t* lenY,
                            int nY, int LY, int d, int dtype,
                            int static_kind, double static_param,
                            int n_levels, int order, int difference,
                            int pairs_mode, const int32_t* pair_list,
                            int n_list, const double* grad_levels, void* dX,
                            double* dparam, void* workspace,
                            size_t workspace_bytes, void* stream);

/*
 * Split gradient pass (no reference counterpart: the reference has no
 * gradients).  The same result as ksig_signature_kern (levels) followed by
 * ksig_signature_kern_bwd (dX, dparam), in two calls that share one
 * workspace: ksig_signature_kern_rec_fwd writes the level kernels
 * ([n_levels + 1, P] float64, level 0 = 1) and keeps, per pair, the records
 * the adjoint needs; ksig_signature_kern_rec_bwd then runs only the adjoint
 * pass.  An autograd forward pays for the records once instead of
 * recomputing the forward recursion in the backward.  The workspace
 * (ksig_signature_kern_rec_workspace bytes: the adjoint's own plus the
 * records, about (L + 33) * n_levels * 128 B per pair in FP32) must stay
 * untouched between the two calls, which take the same arguments.  Order 1
 * (after clamping), n_levels >= 2, difference 1, KSIG_PAIRS_FULL or
 * KSIG_PAIRS_LIST only; ksig_signature_kern_rec_workspace returns 0
 * otherwise.
 */
size_t ksig_signature_kern_rec_workspace(int nX, int LX, int nY, int LY,
                                         int d, int dtype, int n_levels,
                                         int order, int difference,
                                         int pairs_mode, int n_list);
int ksig_signature_kern_rec_fwd(const void* X, const int32_t* lenX, int nX,
                                int LX, const void* Y, const int32_t* lenY,
                                int nY, int LY, int d, int dtype,
                                int static_kind, double static_param,
                                int n_levels, int order, int difference,
                                int pairs_mode, const int32_t* pair_list,
                                int n_list, double* levels, void* workspace,
                                size_t workspace_bytes, void* stream);
int ksig_signature_kern_rec_bwd(const void* X, const int32_t* lenX, int nX,
                                int LX, const void* Y, const int32_t* lenY,
                                int nY, int LY, int d, int dtype,
                                int static_kind, double static_param,
                                int n_levels, int order, int difference,
                                int pairs_mode, const int32_t* pair_list,
                                int n_list, const double* grad_levels,
                                void* dX, double* dparam, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Workspace (bytes) required by ksig_signature_kern_pde_bwd. */
size_t ksig_signature_kern_pde_bwd_workspace(int nX, int LX, int nY, int LY,
                                             int d, int dtype,
                                             int dyadic_order, int difference,
                                             int pairs_mode, int n_list);

/*
 * Adjoint of ksig_signature_kern_pde (no reference counterpart).  For every
 * pair p = (a, b) and grad[p] = dL/dK(p) (float64 [P]) it accumulates
 *   dX[a]   += grad[p] * dK(x_a, y_b) / d x_a   (row side only)
 *   *dparam += grad[p] * dK(x_a, y_b) / d param
 * with the exact discrete adjoint of the Goursat scheme at the given dyadic
 * order.  dX has X's dtype and shape [nX, LX, d] and is not cleared; dparam
 * may be NULL.  difference must be 1.  The workspace holds one refined
 * adjoint grid per resident warp (a few GB at most for long sequences).
 */
int ksig_signature_kern_pde_bwd(const void* X, const int32_t* lenX, int nX,
                                int LX, const void* Y, const int32_t* lenY,
                                int nY, int LY, int d, int dtype,
                                int static_kind, double static_param,
                                int dyadic_order, int difference,
                                int pairs_mode, const int32_t* pair_list,
                                int n_list, const double* grad, void* dX,
                                double* dparam, void* workspace,
                                size_t workspace_bytes, void* stream);

/*
 * Normalisation and level mean (replaces ksig/kernels.py:190-214).
 *   levels   float64 [n_lev, P] from one of the calls above with pairs_mode
 *            FULL (P = nX*nY) or UPPER (P = nX(nX+1)/2, result mirrored).
 *   diagX    float64 [n_lev, nX] per-level K(x_a, x_a) (DIAG call), or NULL
 *            to take the diagonal of `levels` (UPPER, or FULL with X = Y).
 *   diagY    float64 [n_lev, nY], or NULL to reuse diagX.
 *   normalize 1: K_l / (max(sqrt(max(Kx_l, 1e-12)), 1e-12) *
 *            max(sqrt(max(Ky_l, 1e-12)), 1e-12)) then the mean over the
 *            n_lev levels; 0: the sum over levels.
 *   out      [nX, nY] of out_dtype (KSIG_DTYPE_*).
 */
int ksig_normalize_levels(const double* levels, int n_lev, int pairs_mode,
                          int nX, int nY, const double* diagX,
                          const double* diagY, int normalize, void* out,
                          int out_dtype, void* stream);

/*
 * Synchronises `stream`, then reads and clears the device status word that
 * the kernels of the last call on `workspace` wrote (lengths outside [1, L]
 * are clamped and flagged there).  Returns KSIG_OK, KSIG_ERR_INVALID or
 * KSIG_ERR_DEVICE.  No reference counterpart (CuPy raises on the host).
 */
int ksig_workspace_status(void* workspace, void* stream);

/*
 * ksig_workspace_status for the scratch array of ksig_signature_kern_static
 * on the current device (whose address callers cannot see).  Like that
 * entry point, it has no counterpart in the reference.
 */
int ksig_static_status(void* stream);

/*
 * Measurement helpers (no reference counterpart).
 *   ksig_launch_count    kernels launched by this library since it was loaded.
 *   ksig_profile_enable  when on, every main sweep kernel is bracketed by CUDA
 *                        events on its own stream.
 *   ksig_profile_read    waits for the recorded events and returns the summed
 *                        kernel time (ms) and the number of timed launches
 *                        since the last read.
 *   ksig_fp32_peak       measures this GPU's FP32 FMA throughput (TFLOP/s,
 *                        2 flops per FMA) with an FMA-chain kernel on `stream`
 *                        (synchronous).
 */
/*
 * Autotuning hook (no reference counterpart).  Sets the column count per
 * lane (tile width) that later plans of one kernel family prefer:
 * op 0 = DP forward, 1 = PDE forward, 2 = DP adjoint, 3 = PDE adjoint;
 * cols 0 restores the built-in choice.  The nearest compiled width is used.
 * Process-wide; the Python autotuner (ksig_b200.tuning) times the compiled
 * widths on the caller's workload and sets the fastest.
 */
int ksig_tune_set_cols(int op, int cols);
int ksig_tune_get_cols(int op);

unsigned long long ksig_launch_count(void);
void ksig_profile_enable(int on);
int ksig_profile_read(double* total_ms, long long* launches);
int ksig_fp32_peak(double* tflops, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* KSIG_B200_H_ */
