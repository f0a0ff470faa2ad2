/*
 * sigk.h -- C ABI of libsigk.so, the B200 (sm_100a) signature-kernel engine.
 *
 * The library solves the Goursat PDE of the untruncated signature kernel
 * (Salvi et al. 2021) on a dyadically refined grid, and the per-path
 * Chandrupatla root-find of the robust (tensor-normalised) signature kernel
 * (Chevyrev & Oberhauser 2022).  It is the native back end of the
 * `sigpde_b200.torch` package, which keeps stojl/SigPDE's `sigpde.torch` API.
 *
 * Conventions shared by every entry point
 *   - Pointers are DEVICE pointers unless a name says otherwise.  Paths are
 *     C-contiguous (count, length, dim) arrays of `dtype`; outputs are written
 *     in `dtype` too (the reference returns results in the dtype of x).
 *   - Nothing is allocated.  Scratch, when an entry point needs it, comes from
 *     the caller through (workspace, workspace_bytes); sigk_workspace_size()
 *     returns the byte count.  A NULL workspace with workspace_bytes == 0 is
 *     valid whenever the size query returns 0.
 *   - Work is enqueued asynchronously on `stream` (a cudaStream_t; 0 is the
 *     legacy default stream).  No entry point synchronises the device.
 *   - Every entry point returns a sigk_status; sigk_last_error_string() holds
 *     a description of the last failure on the calling host thread.
 *   - Entry points are re-entrant and thread-safe; concurrent calls on
 *     different streams with disjoint outputs and workspaces do not interact.
 *
 * Precision modes (sigk_precision)
 *   SIGK_PREC_FP64  increments <dx_i,dy_j> and PDE cells in float64 (default;
 *                   no worse than the reference's GPU path, which does float64
 *                   arithmetic with float32 storage, and far better).
 *   SIGK_PREC_FP32  increments and cells in float32 (its error grows with |K|
 *                   along the grid and is reported by the tests).
 *   SIGK_PREC_TC32  linear-kernel increments of all pairs from one tensor-core
 *   SIGK_PREC_TC64  GEMM in split TF32 (hi*hi + hi*lo + lo*hi, float32
 *                   accumulate; ~1e-6 relative per increment), stored as a
 *                   float32 matrix in the workspace and read by the wavefront;
 *                   cells in float32 (TC32) or float64 (TC64).  Applies to
 *                   sigk_pairwise / sigk_gram / sigk_gram_sym with dim <= 32
 *                   and to sigk_pairwise_ragged_tc; larger dims, the *_inc,
 *                   sigk_pairwise_ragged and normalisation entry points form
 *                   increments on the CUDA cores with the same cell
 *                   precision.  The workspace holds
 *                   the increment matrix: up to 6 GiB per call (1 GiB at
 *                   order 1 with at most 128 refined rows, where smaller
 *                   chunks read faster; the x paths are processed in chunks
 *                   beyond that; SIGK_TC_CHUNK_MB sets the chunk size).
 *                   Exception: sigk_gram with TC64 at
 *                   order 2 or 3, x paths of one band and dim <= 8 (<= 32 at
 *                   up to 2 coarse rows a lane) runs one fused kernel that
 *                   hands the increments from TMEM through shared memory to
 *                   the wavefront; its workspace holds only the operand
 *                   images, and its results are bitwise those of the
 *                   matrix route (SIGK_FUSED_TC=1: also at orders 0-1;
 *                   SIGK_FUSED_TC=0: never).
 */
#ifndef SIGK_H_
#define SIGK_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(SIGK_BUILD) && defined(__GNUC__)
#define SIGK_API __attribute__((visibility("default")))
#else
#define SIGK_API
#endif

typedef void *sigk_stream_t; /* cudaStream_t */

typedef enum {
    SIGK_OK = 0,
    SIGK_EINVAL = 1,      /* bad argument (shape, dtype, pointer, size)            */
    SIGK_ENOMEM = 2,      /* workspace too small                                   */
    SIGK_ETIMEDOUT = 3,   /* a bounded device wait gave up                         */
    SIGK_ELAUNCH = 4,     /* CUDA launch or runtime error                          */
    SIGK_EUNSUPPORTED = 5 /* valid request that this build does not implement      */
} sigk_status;

typedef enum { SIGK_F32 = 0, SIGK_F64 = 1 } sigk_dtype;

typedef enum { SIGK_PREC_FP64 = 0, SIGK_PREC_FP32 = 1, SIGK_PREC_TC32 = 2, SIGK_PREC_TC64 = 3 } sigk_precision;

/* Static kernels that sigk_gram_static evaluates on the device
 * (sigpde/torch/static_kernels.py:3-53); param is LinearKernel's scale or the
 * RBF kernels' sigma. */
typedef enum { SIGK_STATIC_LINEAR = 0, SIGK_STATIC_RBF = 1, SIGK_STATIC_L1RBF = 2 } sigk_static_kind;

typedef enum {
    SIGK_OP_PAIRWISE = 0,     /* out[b]    = k(x_b, y_b)                                */
    SIGK_OP_GRAM = 1,         /* out[i][j] = k(x_i, y_j)                                */
    SIGK_OP_GRAM_SYM = 2,     /* out[i][j] = k(x_i, x_j), lower triangle solved, mirrored */
    SIGK_OP_NORMALIZE = 3     /* robust lambda per path                                 */
} sigk_op;

/* Library version string, e.g. "sigk 0.1.0 sm_100a". */
SIGK_API const char *sigk_version(void);

/* Description of the last error on this host thread ("" if none). */
SIGK_API const char *sigk_last_error_string(void);

/* Number of kernels this library has enqueued since it was loaded (all
 * threads, all devices); a caller can difference it around a region. */
SIGK_API uint64_t sigk_launch_count(void);

/*
 * Bound of the uneven-batch kernels' band waits (a band of a pair waits for
 * the band above it to publish its bottom row, sigk_pairwise_ragged*): a
 * wait gives up after `polls` polls of ~64 ns each, sets the timeout bit of
 * the launch's error word and the pair's result becomes NaN; the kernel
 * still returns.  polls < 0 restores the default (2^26 polls, ~4 s); 0 gives
 * up at the first poll that finds nothing published.  Applies to launches
 * enqueued afterwards, from every thread; returns the previous setting (-1 for
 * the default).  It has no counterpart in the reference, whose kernels have
 * no waits; it exists so that the timeout path can be exercised on purpose.
 */
SIGK_API int64_t sigk_set_wait_limit(int64_t polls);

/*
 * Bytes of caller-provided scratch an entry point needs for the given shape.
 * `op` is a sigk_op; len_x / len_y are path lengths before refinement; for
 * SIGK_OP_PAIRWISE n_x is the batch, for the Gram ops n_x / n_y are the path
 * counts.  Pass dim = 0 for the *_inc entry points (len_x / len_y are then
 * nc_x + 1 / nc_y + 1).  Returns 0 when no scratch is needed.  The size
 * depends on the current device's SM count.
 */
SIGK_API size_t sigk_workspace_size(int op, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y, int64_t dim,
                           int order, int dtype, int precision);

/*
 * Pairwise signature kernel with the linear static kernel.
 * Replaces SigPDE.pairwise's increment build + PairwisePDESolver.solve /
 * solve_scaled (sigpde/torch/kernel.py:31-65, sigpde/torch/kernel.py:13-16,
 * sigpde/PDESolvers.py:56-84, sigpde/cuda_pairwise_kernels.py:8-85).
 *   x: (batch, len_x, dim), y: (batch, len_y, dim); out: (batch,)
 *   static_scale: LinearKernel(scale) factor (sigpde/torch/static_kernels.py:4-8)
 *   scale_x / scale_y: (batch,) per-pair path scales or NULL (NULL = 1)
 */
SIGK_API int sigk_pairwise(const void *x, const void *y, int64_t batch, int64_t len_x, int64_t len_y, int64_t dim,
                  int dtype, int order, double static_scale, const void *scale_x, const void *scale_y, void *out,
                  int precision, void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Gram matrix with the linear static kernel.
 * Replaces SigPDE._gram's tile loop, gram_inner_product and
 * GramPDESolver.solve / solve_scaled (sigpde/torch/kernel.py:75-126,
 * sigpde/torch/kernel.py:18-21, sigpde/PDESolvers.py:160-190,
 * sigpde/cuda_gram_kernels.py:8-76).
 *   x: (n_x, len_x, dim), y: (n_y, len_y, dim); out: (n_x, n_y) row-major
 *   scale_x: (n_x,) or NULL, scale_y: (n_y,) or NULL
 */
SIGK_API int sigk_gram(const void *x, const void *y, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y, int64_t dim,
              int dtype, int order, double static_scale, const void *scale_x, const void *scale_y, void *out,
              int precision, void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Symmetric Gram matrix k(x_i, x_j): only the lower triangle i >= j is solved
 * and each entry is written to [i][j] and [j][i].
 * Replaces SigPDE._gram_sym + SymmetricGramPDESolver.solve / solve_scaled
 * (sigpde/torch/kernel.py:128-171, sigpde/PDESolvers.py:192-245,
 * sigpde/cuda_gram_kernels.py:79-164).
 *   x: (n, len, dim); scale: (n,) or NULL; out: (n, n)
 */
SIGK_API int sigk_gram_sym(const void *x, int64_t n, int64_t len, int64_t dim, int dtype, int order, double static_scale,
                  const void *scale, void *out, int precision, void *workspace, size_t workspace_bytes,
                  sigk_stream_t stream);

/*
 * Gram matrix (op = SIGK_OP_GRAM) or symmetric Gram (op = SIGK_OP_GRAM_SYM,
 * y = NULL, n_y / len_y / scale_y ignored) with a static kernel evaluated from
 * the path points on the device:
 *   SIGK_STATIC_LINEAR  param * <x, y>: the sigk_gram / sigk_gram_sym path;
 *   SIGK_STATIC_RBF     exp(-(|x|^2 + |y|^2 - 2<x, y>) / param);
 *   SIGK_STATIC_L1RBF   exp(-|x - y|_1 / param).
 * Replaces, for RBFKernel / L1RBFKernel, SigPDE._gram / _gram_sym's tile loop
 * with the static Gram, the 4-term difference and the solver
 * (sigpde/torch/kernel.py:18-21,75-171, sigpde/torch/static_kernels.py:13-53,
 * sigpde/cuda_gram_kernels.py:8-164).  The static Gram is evaluated in
 * float64 (the reference uses the input dtype) and each increment is written
 * once to a matrix in the workspace, which the wavefront reads: float64 for
 * float64 cells (SIGK_PREC_FP64 / SIGK_PREC_TC64), rounded once to float32
 * for float32 cells (SIGK_PREC_FP32 / SIGK_PREC_TC32).  dim <= 32
 * (SIGK_EUNSUPPORTED otherwise: sigk_gram_inc takes any increments).
 * Workspace: sigk_static_workspace_size(op, kind, ...) bytes, 256-byte
 * aligned.
 */
SIGK_API size_t sigk_static_workspace_size(int op, int kind, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y,
                                           int64_t dim, int order, int dtype, int precision);
SIGK_API int sigk_gram_static(int op, int kind, double param, const void *x, const void *y, int64_t n_x, int64_t n_y,
                              int64_t len_x, int64_t len_y, int64_t dim, int dtype, int order, const void *scale_x,
                              const void *scale_y, void *out, int precision, void *workspace,
                              size_t workspace_bytes, sigk_stream_t stream);

/*
 * Backward pass (no counterpart in the reference, whose Numba kernels end
 * autograd): gradients of  L = sum_b grad_out[b] k(x_b, y_b)  (op =
 * SIGK_OP_PAIRWISE, n_y = n_x) or  L = sum_ij grad_out[i][j] k(x_i, y_j)
 * (op = SIGK_OP_GRAM) with respect to the points of x and y, for the linear
 * static kernel (static_scale) with per-path scales scale_x / scale_y (held
 * constant), by the adjoint of the float64 scheme.
 *   grad_out: (n_x,) or (n_x, n_y) row-major, in dtype
 *   grad_x: (n_x, len_x, dim), grad_y: (n_y, len_y, dim), in dtype; either may
 *   be NULL (not computed).  For a symmetric Gram pass y = x and add the two.
 * Dyadic order <= 4 (SIGK_EUNSUPPORTED above).  Workspace:
 * sigk_backward_workspace_size(...) bytes, 256-byte aligned (pairs are taken
 * in chunks of x paths so that it stays near 8 GiB plus the inputs' size).
 */
SIGK_API size_t sigk_backward_workspace_size(int op, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y,
                                             int64_t dim, int order, int dtype);
SIGK_API int sigk_backward(int op, const void *x, const void *y, int64_t n_x, int64_t n_y, int64_t len_x,
                           int64_t len_y, int64_t dim, int dtype, int order, double static_scale,
                           const void *scale_x, const void *scale_y, const void *grad_out, void *grad_x,
                           void *grad_y, void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Backward pass over caller's increments (any static kernel): for
 * L = sum_b grad_out[b] k_b, where k_b solves the PDE on increments
 * inc[b] * scale_x[b] * scale_y[b] as sigk_pairwise_inc does, writes
 * grad_inc = dL/dinc (npairs, nc_x, nc_y) with element strides (g0, g1, g2)
 * in dtype.  A Gram tile passes its pairs flattened (strides of the 4-D
 * tensor's last two axes, s0 = the stride between consecutive pairs when they
 * are evenly spaced, else one call per row).  Float64 adjoint; dyadic order
 * <= 4.  Workspace: sigk_backward_inc_workspace_size(...) bytes, 256-byte
 * aligned.  No counterpart in the reference.
 */
SIGK_API size_t sigk_backward_inc_workspace_size(int64_t npairs, int64_t nc_x, int64_t nc_y, int order);
SIGK_API int sigk_backward_inc(const void *inc, int64_t npairs, int64_t nc_x, int64_t nc_y, int64_t s0, int64_t s1,
                               int64_t s2, int dtype, int order, const void *scale_x, const void *scale_y,
                               const void *grad_out, void *grad_inc, int64_t g0, int64_t g1, int64_t g2,
                               void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Self norms k(x_b, x_b) in float64, NaN mapped to +inf.
 * First half of RobustSigPDE._norm_factors (sigpde/torch/kernel.py:181-183);
 * used when the normaliser is a user callable that the host applies.
 *   x: (n, len, dim); knorm: (n,) float64
 */
SIGK_API int sigk_self_norms(const void *x, int64_t n, int64_t len, int64_t dim, int dtype, int order, double static_scale,
                    double *knorm, void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Robust normalisation lambda per path: the Chandrupatla root-find of
 * g(l) = k(l x, l x) - f(k(x,x)) on [0,1], every iteration re-solving the PDE
 * on-chip with float64 cells and float64 bracket arithmetic, then lambda = 0
 * where k(x,x) < 1.
 * Replaces RobustSigPDE._norm_factors + PairwisePDESolver.solve_norms
 * (sigpde/torch/kernel.py:180-195, sigpde/PDESolvers.py:86-101,
 * sigpde/cuda_pairwise_kernels.py:88-165).
 *   fnorm == NULL: the default normaliser f(s) = 2 - 1/(1 + log s)
 *                  (sigpde/torch/kernel.py:23-24) is applied on the device and
 *                  knorm receives k(x,x) (if knorm != NULL).
 *   fnorm != NULL: knorm (input, float64, from sigk_self_norms) and fnorm
 *                  (input, float64, f(knorm) computed by the caller) are used.
 *   lam: (n,) in dtype.  iters (int32, may be NULL) receives iteration counts.
 */
SIGK_API int sigk_normalize(const void *x, int64_t n, int64_t len, int64_t dim, int dtype, int order, double static_scale,
                   double *knorm, const double *fnorm, double tol, int maxit, void *lam, int *iters,
                   void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Generic-increment entry points, for static kernels other than the linear
 * one (RBF, L1-RBF, any duck-typed kernel).  The caller computes the coarse
 * increments (the 4-term second difference of the static Gram divided by
 * 4^order, sigpde/torch/kernel.py:13-21) and the library solves the PDE.
 *
 * sigk_pairwise_inc replaces PairwisePDESolver.solve / solve_scaled
 * (sigpde/PDESolvers.py:56-84):
 *   inc: (batch, nc_x, nc_y) with element strides (s0, s1, s2); out: (batch,)
 */
SIGK_API int sigk_pairwise_inc(const void *inc, int64_t batch, int64_t nc_x, int64_t nc_y, int64_t s0, int64_t s1, int64_t s2,
                      int dtype, int order, const void *scale_x, const void *scale_y, void *out, int precision,
                      void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * sigk_gram_inc replaces GramPDESolver.solve / solve_scaled and, with
 * symmetric != 0, SymmetricGramPDESolver.solve / solve_scaled
 * (sigpde/PDESolvers.py:160-245):
 *   inc: (n_x, n_y, nc_x, nc_y) with element strides (s0, s1, s2, s3);
 *   out: (n_x, n_y) row-major with row stride out_ld (elements).
 *   symmetric: solve only i >= j and mirror (requires n_x == n_y).
 */
SIGK_API int sigk_gram_inc(const void *inc, int64_t n_x, int64_t n_y, int64_t nc_x, int64_t nc_y, int64_t s0, int64_t s1,
                  int64_t s2, int64_t s3, int dtype, int order, const void *scale_x, const void *scale_y,
                  int symmetric, void *out, int64_t out_ld, int precision, void *workspace, size_t workspace_bytes,
                  sigk_stream_t stream);

/*
 * sigk_normalize_inc replaces PairwisePDESolver.solve_norms
 * (sigpde/PDESolvers.py:86-101, sigpde/cuda_pairwise_kernels.py:88-165) for
 * precomputed self-increments inc: (n, nc, nc) with strides (s0, s1, s2).
 * knorm and fnorm are float64 inputs (k(x,x) and f(k(x,x))).
 */
SIGK_API int sigk_normalize_inc(const void *inc, int64_t n, int64_t nc, int64_t s0, int64_t s1, int64_t s2, int dtype,
                       int order, const double *knorm, const double *fnorm, double tol, int maxit, void *lam,
                       int *iters, void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Uneven batched pairwise signature kernels: pair b compares x path b and
 * y path b, each of its own length, at its own dyadic order, in one launch.
 * No reference call covers this: the reference needs one SigPDE.pairwise call
 * per (length_x, length_y, order) bucket (sigpde/torch/kernel.py:31-65).
 *   x_pack: all x paths' points back to back, (x_points, dim) in dtype, with
 *         x_points = sum_b x_len[b] (every path >= 2 points);
 *   x_off[b], x_len[b] (int64, device): first point and length of x path b;
 *         they must describe x_pack (x_off[b] = x_len[0] + ... + x_len[b-1]);
 *   y_pack, y_off, y_len, y_points: the same for y;  order[b] (int32, device).
 * The work plan (device arrays, built once per batch shape, see
 * sigpde_b200/torch/ragged.py): with n_b = (min(x_len,y_len) - 1) << order and
 * m_b = (max(x_len,y_len) - 1) << order,
 *   pair_rows[b]  in {2, 4, 8, 16}: rows per lane;
 *   pair_bands[b] = ceil(n_b / (32 * pair_rows[b]));
 *   pair_bnd_off[b]: offset (cell-type elements) of the pair's
 *         (pair_bands[b] - 1) * (m_b + 1) boundary values in a pool of bnd_elems;
 *   item_pair[i], item_band[i] (nitems items): every band of every pair, the
 *         bands of a pair consecutive and in increasing order, pairs in the
 *         order they should start (longest first balances best).
 * An item that breaks these rules (or an order outside [0, 12]) gives NaN for
 * its pair and is not solved.  scale_x, scale_y: (npairs,) or NULL;
 * out: (npairs,) in dtype.
 * Workspace: sigk_ragged_workspace_size(npairs, x_points, y_points, dim,
 * nitems, bnd_elems, precision) bytes, 256-byte aligned.
 */
SIGK_API size_t sigk_ragged_workspace_size(int64_t npairs, int64_t x_points, int64_t y_points, int64_t dim,
                                           int64_t nitems, int64_t bnd_elems, int precision);
SIGK_API int sigk_pairwise_ragged(const void *x_pack, const int64_t *x_off, const int64_t *x_len, int64_t x_points,
                                  const void *y_pack, const int64_t *y_off, const int64_t *y_len, int64_t y_points,
                                  const int *order, const int64_t *item_pair, const int *item_band, int64_t nitems,
                                  const int *pair_rows, const int *pair_bands, const int64_t *pair_bnd_off,
                                  int64_t bnd_elems, int64_t npairs, int64_t dim, int dtype, double static_scale,
                                  const void *scale_x, const void *scale_y, void *out, int precision,
                                  void *workspace, size_t workspace_bytes, sigk_stream_t stream);

/*
 * Precomputed increments for an uneven batch: tensor cores (precision
 * SIGK_PREC_TC32 or SIGK_PREC_TC64, dim <= 32), or, with SIGK_PREC_FP64 (any
 * dim), float64 increments from one FP64 GEMM on the CUDA cores over the same
 * plan's tiles into float64 blocks (offsets and ld in doubles).  Pair b's coarse increments
 * <d row_ci, d col_cj> (row path = the shorter of its two paths, as the
 * wavefront puts it on the rows; rows_b = its coarse cells, cols_b the other
 * path's) come from one grouped split-TF32 tcgen05 GEMM into a float32 block
 * of cols_b columns of ld_b = round_up(rows_b, 4) floats, which the wavefront
 * then reads.  The plan (device arrays except the counts, built once per batch
 * shape, see sigpde_b200/torch/ragged.py):
 *   a_row0[b]: first row of pair b's row path in the A operand image (a
 *     multiple of 8, the pair taking round_up(rows_b, 8) rows); a_rows: image
 *     rows, at least the last pair's end + 128;
 *   b_row0[b], b_rows: the same for the column paths (end + N, N below);
 *   inc_off[b]: offset (floats, a multiple of 4) of pair b's block in a matrix
 *     of inc_elems floats;
 *   tile_n: 0 or 256 for 128 x 256 GEMM tiles, 128 for 128 x 128 tiles
 *     (tensor-core precisions only; an autotuner knob, same results); with
 *     N = tile_n (256 when 0) and b_rows >= the last pair's end + N:
 *   tiles (ntiles x 6 int64): one 128 x N GEMM tile each,
 *     {a_row, b_row, m_valid, n_valid, out_off, ld}: a_row = a_row0[b] + 128 i,
 *     b_row = b_row0[b] + N j, m_valid = min(128, rows_b - 128 i),
 *     n_valid = min(N, cols_b - N j), out_off = inc_off[b] + N j ld_b +
 *     128 i, ld = ld_b, for every tile (i, j) of every pair.
 * A tile entry outside these buffers is skipped and the affected pairs give
 * NaN (with the error flag of the ragged launch set).  The remaining
 * arguments are those of sigk_pairwise_ragged.  Workspace:
 * sigk_ragged_tc_workspace_size(npairs, dim, nitems, bnd_elems, precision,
 * &plan) bytes, 256-byte aligned.
 */
typedef struct {
    const int64_t *a_row0;
    const int64_t *b_row0;
    int64_t a_rows;
    int64_t b_rows;
    const int64_t *inc_off;
    int64_t inc_elems;
    const int64_t *tiles;
    int64_t ntiles;
    int64_t tile_n;
} sigk_ragged_tc_plan;

SIGK_API size_t sigk_ragged_tc_workspace_size(int64_t npairs, int64_t dim, int64_t nitems, int64_t bnd_elems,
                                              int precision, const sigk_ragged_tc_plan *plan);
SIGK_API int sigk_pairwise_ragged_tc(const void *x_pack, const int64_t *x_off, const int64_t *x_len,
                                     int64_t x_points, const void *y_pack, const int64_t *y_off,
                                     const int64_t *y_len, int64_t y_points, const int *order,
                                     const int64_t *item_pair, const int *item_band, int64_t nitems,
                                     const int *pair_rows, const int *pair_bands, const int64_t *pair_bnd_off,
                                     int64_t bnd_elems, int64_t npairs, int64_t dim, int dtype, double static_scale,
                                     const void *scale_x, const void *scale_y, void *out, int precision,
                                     const sigk_ragged_tc_plan *plan, void *workspace, size_t workspace_bytes,
                                     sigk_stream_t stream);

/*
 * Outcome of the last uneven-batch launch that used `workspace`: synchronises
 * `stream`, then reads the launch's error word.  SIGK_ETIMEDOUT: a band wait
 * ran out (see sigk_set_wait_limit) or the increment GEMM gave up a wait;
 * SIGK_EINVAL: an item broke the plan rules; either way those pairs are NaN
 * and the others are exact.  The device and the library stay usable.
 * The reference reports failures as NaN -> inf in its results only
 * (sigpde/torch/kernel.py:183, sigpde/cuda_pairwise_kernels.py:132).
 */
SIGK_API int sigk_ragged_status(const void *workspace, sigk_stream_t stream);

/*
 * sigk_gram_noalloc -- sigk_gram for callers that cannot allocate device
 * memory.  It has no counterpart in the reference.
 *
 * Same arguments and result as sigk_gram, minus the workspace: the scratch
 * sigk_gram takes from the caller comes from an 8 MiB array that is part of
 * this library's device image (each GPU that loads the library holds it until
 * the process exits).  Nothing is allocated.  A Gram whose scratch
 * (sigk_workspace_size(SIGK_OP_GRAM, ...)) exceeds 8 MiB is rejected with
 * SIGK_EINVAL and a message naming the limit; 256 x 256 paths of length 128
 * in 8 dimensions at order 2 with float64 cells need about 4.2 MB.
 *
 * The first call on a device looks up the array's device address (with that
 * device current) and caches it; make that first call before any stream
 * capture.  The cached address belongs to the device's primary context: after
 * cudaDeviceReset the array is loaded again, possibly elsewhere, and this entry
 * point must not be called again in that process.
 * Every call shares the one array and leaves its contents behind;
 * each call overwrites the part it reads before reading it.  Calls that
 * overlap on the GPU (two streams, or two host threads, on one device) race on
 * the array: serialise them.
 */
SIGK_API int sigk_gram_noalloc(const void *x, const void *y, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y,
                               int64_t dim, int dtype, int order, double static_scale, const void *scale_x,
                               const void *scale_y, void *out, int precision, sigk_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SIGK_H_ */
