/*
 * cfb200.h - C ABI of libcfb200.so, the B200 (sm_100a) device library for
 * CosmoForge's pixel-space QML / Fisher / pixel-likelihood path.
 *
 * Conventions
 *   - Every pointer argument named as a matrix / vector / table is a DEVICE
 *     pointer (allocated by the caller, e.g. with PyTorch or cudaMalloc).
 *   - Matrices are row-major FP64 with an explicit leading dimension (ld,
 *     in elements); batched calls take element strides between problems.
 *   - `stream` is a cudaStream_t passed as void*; calls are asynchronous on
 *     it unless stated.
 *   - Return value: CF_OK (0) or a negative CF_ERR_* code.  Per-problem
 *     numerical status (non positive-definite pivots) is written to a
 *     device `info` array, LAPACK style: 0 ok, k > 0 the leading minor of
 *     order k is not positive.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   cosmocore/signal_kernels.py      signal_matrix, compute_signal_matrix,
 *                                    compute_00/22/02_contribution, do_derivative_step
 *   cosmocore/basis/pixel.py         PixelBasis.get_binned_derivative_direct
 *   cosmocore/basics/linalg.py       matrix_inverse_symm, cholesky_factor,
 *                                    matrix_slogdet_symm, matrix_trace, matrix_mult
 *   qube/fisher.py                   Fisher.compute (A_b and trace loops)
 *   qube/spectra.py                  Spectra._compute_qml_spectra_traditional
 *   picslike/picslike.py             PICSLike._compute_likelihood_point
 */
#ifndef CFB200_H
#define CFB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CF_OK 0
#define CF_ERR_ARG -1         /* invalid argument */
#define CF_ERR_CUDA -2        /* a kernel launch or CUDA runtime call failed */
#define CF_ERR_TIMEOUT -3     /* a bounded device wait ran out */
#define CF_ERR_UNSUPPORTED -4 /* valid but not implemented combination */
#define CF_ERR_TOO_LARGE -5   /* size exceeds a static capacity of the library */

/* Block kinds of cf_build_block (which field pair a block of S couples). */
#define CF_KIND_00_AUTO 0  /* spin-0 field with itself */
#define CF_KIND_00_CROSS 1 /* two different spin-0 fields */
#define CF_KIND_22_AUTO 2  /* spin-2 field with itself: rows/cols [Q | U] */
#define CF_KIND_02 3       /* rows: spin-2 field [Q | U], cols: spin-0 field */

/* Library version (>= 1). */
int cf_version(void);

/* Number of kernels the library has launched so far in this process. */
unsigned long long cf_launch_count(void);

/*
 * Fused pixel-pair builder: one block of the signal matrix S, or the binned
 * derivatives dC_b of every bin of one spectrum, from one pass of the
 * Legendre / spin-2 recurrences per pixel pair.
 * Replaces: cosmocore/signal_kernels.py:164-387 (compute_00/22/02_contribution,
 * the per-pair loops), :390-537 (compute_signal_matrix / signal_matrix),
 * :715-829 (do_derivative_step), cosmocore/basis/pixel.py:802-950
 * (get_binned_derivative_direct).
 *   kind, mode   CF_KIND_*; mode < 0 builds the signal (t0..t2 are the
 *                block's beam-smoothed C_l: 00 -> t0 = C_l; 22 -> EE, BB, EB;
 *                02 -> TE, TB); mode >= 0 builds derivatives of one spectrum
 *                (22: 0 EE, 1 BB, 2 EB; 02: 0 TE, 1 TB) with t0 = w_l b_l^2.
 *   na, va       column field: pixel count and pointings, SoA x[na] y[na] z[na]
 *   nb, vb       row field (== column field for *_AUTO kinds)
 *   lmax         last multipole of the recurrence (<= 512)
 *   bin_of       int[lmax+1]: output bin of each l, -1 = none; NULL = one bin
 *   out, ld, row_off, col_off, bin_stride
 *                entry (r, c) of bin b goes to
 *                out[(row_off + r) * ld + col_off + b * bin_stride + c]
 *   outT, ...    its mirror (c, r) goes to
 *                outT[(rowT_off + c) * ldT + colT_off + b * binT_stride + r]
 *   batch, tstride, ostride
 *                batch of problems: tables advance by tstride, out/outT by ostride
 */
int cf_build_block(int kind, int mode, int na, const double* va, int nb, const double* vb, int lmax,
                   const double* t0, const double* t1, const double* t2, const int* bin_of,
                   double* out, long ld, long row_off, long col_off, long bin_stride, double* outT,
                   long ldT, long rowT_off, long colT_off, long binT_stride, int batch, long tstride,
                   long ostride, void* stream);

/*
 * FP64 GEMM on the DMMA tensor pipe: C = alpha op(A) op(B) + beta C, with an
 * optional transposed copy CT = C^T (NULL to skip) and a batch dimension.
 * transa / transb: 0 = A is M x K / B is K x N; 1 = A given as K x M / B as N x K.
 * lower_only: bit 0 skips output tiles strictly above the diagonal; bit 1
 * starts each tile's K sum at its first row (op(A) upper triangular, e.g.
 * op(A) = Y^T with Y lower); bit 2 ends it after its last row (op(A) lower
 * triangular).  Bits 1 and 2 assume M == K (a square triangular op(A)).
 * Bit 3 treats batch entry z as row z of a symmetric block and skips the
 * output tiles that start right of column z (the lower triangle of a block
 * built row by row; entries right of z inside a computed tile are written too).
 * Replaces: cosmocore/basics/linalg.py:18-32 (matrix_mult, np.matmul).
 */
int cf_dgemm(int transa, int transb, int M, int N, int K, double alpha, const double* A, long lda,
             long strideA, const double* B, long ldb, long strideB, double beta, double* C, long ldc,
             long strideC, double* CT, long ldct, long strideCT, int batch, int lower_only,
             void* stream);

/*
 * cf_dgemm with a rounded FP32 copy of the result (C32: row stride ldc32,
 * batch stride strideC32) written by the same epilogue in place of CT, so an
 * FP64 matrix and its FP32 copy come out of one pass.  Used to build the
 * mixed likelihood's C(theta) (FP64 for the refinement, FP32 to factor).
 * Replaces: the per-point covariance build of picslike/picslike.py:301-319
 * with its FP32 cast, in the mixed likelihood.
 */
int cf_dgemm_f32copy(int transa, int transb, int M, int N, int K, double alpha, const double* A, long lda,
                     long strideA, const double* B, long ldb, long strideB, double beta, double* C, long ldc,
                     long strideC, float* C32, long ldc32, long strideC32, int batch, int lower_only,
                     void* stream);

/* Bytes of workspace cf_potrf needs for `batch` problems of order n. */
size_t cf_potrf_workspace(int n, int batch);

/* Doubles between consecutive problems' diagonal-block inverses in the
 * cf_potrf workspace (block j of problem z at work + z stride + j 64^2, row
 * major with row stride kb_j).  No counterpart in the reference. */
size_t cf_potrf_dinv_stride(int n);

/*
 * Blocked lower Cholesky factorisation in place (batch of n x n matrices):
 * 64-wide panels, diagonal block factored and inverted by one CTA, panel and
 * trailing updates as DMMA GEMMs.  A single matrix (batch 1) of order above
 * 1024 is factored with a look-ahead: the critical path runs on an internal
 * high-priority stream forked from and joined back to `stream` by events
 * (stream-ordered, capturable into a CUDA graph), the bulk of each trailing
 * update on `stream`.  work: cf_potrf_workspace(n, batch) bytes (keeps the
 * diagonal-block inverses for cf_trtri_lower; one more panel buffer for the
 * look-ahead).  info: int[batch], zeroed by the caller.
 * Replaces: cosmocore/basics/linalg.py:362-406 (cholesky_factor, LAPACK dpotrf).
 */
int cf_potrf(int n, double* A, long lda, long strideA, int batch, void* work, int* info, void* stream);

/* Y = L^-1 for the lower factor L of a preceding cf_potrf with the same `work`
 * (batch).  Replaces the dpotri half of cosmocore/basics/linalg.py:152-219. */
int cf_trtri_lower(int n, const double* L, long lda, long strideL, double* Y, long ldy, long strideY,
                   int batch, void* work, void* stream);

/* Bytes of workspace cf_spd_inverse needs for `batch` problems of order n. */
size_t cf_spd_inverse_workspace(int n, int batch);

/*
 * In place inverse of SPD matrices with the reference's Jacobi scaling:
 * D = diag(|A_ii|^-1/2), L L^T = D A D, A^-1 = D (L L^T)^-1 D.
 * work: cf_spd_inverse_workspace(n, batch) bytes of device memory.
 * Replaces: cosmocore/basics/linalg.py:152-219 (matrix_inverse_symm).
 */
int cf_spd_inverse(int n, double* A, long lda, long strideA, int batch, void* work, int* info,
                   void* stream);

/*
 * Allocation-free SPD inverse: cf_spd_inverse for one n x n matrix whose
 * workspace is a scratch array compiled into the library (a file-scope
 * __device__ array of 1.25 M doubles, 10.0 MB per device).  It serves
 * callers that must not allocate device memory at the point where they need
 * the inverse: allocator hooks, plugins whose host application owns the
 * memory pool and forbids allocations after start-up, and integrations that
 * must not fragment a pool they do not own.  It launches kernels and makes
 * CUDA runtime calls, so it must not be called from inside a host callback
 * (cudaLaunchHostFunc, cudaStreamAddCallback), where CUDA calls are not
 * permitted.  With lazy module loading (the CUDA 12 default) a device
 * allocates the array when the module that holds it is first used there,
 * and the first call on a device also looks up the array's address
 * (cudaGetSymbolAddress) and sets kernel attributes: make one warm-up call
 * per device at start-up, outside the no-allocation context and before any
 * stream capture; later calls allocate nothing.
 * n > cf_spd_inverse_static_max_n() returns CF_ERR_TOO_LARGE.  All calls
 * share the one array: calls that overlap on the GPU race.  *info is zeroed
 * on `stream` by the call.
 * No counterpart in the reference (an addition of this library).
 */
int cf_spd_inverse_static(int n, double* A, long lda, int* info, void* stream);

/* Largest n accepted by cf_spd_inverse_static. */
int cf_spd_inverse_static_max_n(void);

/*
 * Fisher trace contraction, split-K on the DMMA pipe:
 *   F[(p_off+p) ldF + q_off+q] += scale sum_{k<K1, l<K2} X[p sXp + k ldX + l] Y[q sYq + k ldY + l]
 * (and the mirror entry when sym != 0), p < P1, q < P2.  F must be zeroed
 * first; splits <= 0 picks 4 CTAs per SM.
 * Replaces: qube/fisher.py:557-607 (trace loop), cosmocore/basics/linalg.py:66-98
 * (matrix_trace).
 */
int cf_trace_contract_f64(int P1, int P2, int K1, int K2, const double* X, long sXp, long ldX,
                          const double* Y, long sYq, long ldY, double scale, double* F, long ldF,
                          long p_off, long q_off, int sym, int splits, void* stream);

/*
 * QML reductions over the derivative blocks D_p (R x Ccols, p-th block at
 * D + p sDp, row stride ldD) of one spectrum:
 *   bias[p] += scale sum_{r,c} M[(mro+r) ldM + mco+c] D_p[r, c]            (M may be NULL)
 *   q[m ldq + p] += scale sum_{r,c} Y[(yro+r) ldY + m] D_p[r, c] Y[(yco+c) ldY + m],  m < nsims <= 4
 * Replaces: qube/spectra.py:1124-1186 (q_b = y^T dC_b y / 2, bias_b = Tr(C^-1 N C^-1 dC_b) / 2).
 */
int cf_qml_reduce_f64(int P, int R, int Ccols, const double* D, long ldD, long sDp, const double* M,
                      long ldM, long mro, long mco, const double* Y, long ldY, int nsims, long yro,
                      long yco, double scale, double* bias, double* q, long ldq, void* stream);

/*
 * chi2[b nrhs + m] = |L_b^-1 x_{b,m}|^2 and logdet[b] = 2 sum ln (L_b)_ii
 * from lower Cholesky factors (batch).  X: n x nrhs (ldx), strideX = 0 shares
 * it across the batch; z_work: batch * nrhs * n doubles, used (and required)
 * only for n > 24576, may be NULL below (the solve vector lives in shared
 * memory).
 * Replaces: picslike/picslike.py:643-664 (chi2 einsum with C^-1) and
 * cosmocore/basics/linalg.py:430-474 (matrix_slogdet_symm).
 */
int cf_chi2_logdet(int n, const double* L, long lda, long strideL, int batch, const double* X, long ldx,
                   long strideX, int nrhs, double* z_work, double* chi2, double* logdet, void* stream);

/* cf_chi2_logdet with the factor's 64 x 64 diagonal-block inverses that
 * cf_potrf leaves in its workspace (Dinv = the workspace, strideD =
 * cf_potrf_dinv_stride(n) doubles between problems): the solve runs over
 * 64-row blocks, each diagonal solve one block-times-vector product instead
 * of a dependent substitution.  n <= 24512.  Same replaced reference code. */
int cf_chi2_logdet_dinv(int n, const double* L, long lda, long strideL, const double* Dinv, long strideD,
                        int batch, const double* X, long ldx, long strideX, int nrhs, double* chi2,
                        double* logdet, void* stream);

/* Z_b = a X_b + c_b W_b (c_b = cvec[b] if cvec else c; strideW = 0 shares W).
 * Used for C = S + s N (picslike/picslike.py:301-319, qube/fisher.py:311-344). */
int cf_axpby(long count, double a, const double* X, long strideX, double c, const double* cvec,
             const double* W, long strideW, double* Z, long strideZ, int batch, void* stream);

/* B = A^T for an R x C row-major A. */
int cf_transpose(int R, int C, const double* A, long lda, double* B, long ldb, void* stream);

/* ---- Mixed-precision path: BF16 split planes on the tcgen05 tensor cores ----
 * An FP64 value x is carried as planes x_0 = bf16(x), x_1 = bf16(x - x_0),
 * x_2 = bf16(x - x_0 - x_1); a product list {(a_t, b_t)} selects which plane
 * pairs are multiplied: BF16x3 = {(0,0),(0,1),(1,0)} (~16 bits), BF16x6 adds
 * {(0,2),(1,1),(2,0)} (~24 bits).  Plane arrays are __nv_bfloat16, passed as
 * void*.  err: device int set to 1 when a bounded wait inside a tensor-core
 * kernel ran out (the kernel then returns early; results are invalid). */

/* BF16 split planes of an R x C FP64 matrix (row stride ldx) into `planes`
 * (1..3) planes of row stride ldo, plane_stride elements apart.  Operand
 * preparation for qube/fisher.py:501-531 (A_b = C^-1 dC_b) in mixed precision. */
int cf_split_bf16(int R, int C, const double* X, long ldx, int planes, void* out, long ldo,
                  long plane_stride, void* stream);

/* BF16 split planes of the outer products x_q y_q^T (n x n, q < nvec; x and y
 * are n x nvec with row stride ldv) into out[p][q] (row stride ld, q_stride /
 * plane_stride elements apart).  The quadratic forms of
 * qube/spectra.py:1124-1186 as contractions against resident A_b slabs. */
int cf_outer_planes(int n, int nvec, const double* x, const double* y, long ldv, int planes, void* out,
                    long ld, long q_stride, long plane_stride, void* stream);

/* As cf_outer_planes for m x n products: x is m x nvec, y is n x nvec (row
 * stride ldv), out[p][q] is m x n.  The mixed Fisher appends y_q x_q^T and
 * C^-1 N to the A_b slabs as extra contraction partners, so one pass of the
 * trace kernel gives F, the noise bias and the quadratic forms
 * (qube/fisher.py:501-607, qube/spectra.py:1124-1186). */
int cf_outer_planes_rect(int m, int n, int nvec, const double* x, const double* y, long ldv, int planes,
                         void* out, long ld, long q_stride, long plane_stride, void* stream);

/* cf_build_block writing BF16 split planes (planes 1..3, plane_stride /
 * planeT_stride elements apart) instead of FP64.  flags bit 0 (auto kinds):
 * every entry computed from its own pixel pair, no mirror writes; bit 1
 * (cross kinds): write only the transposed block outT.  Replaces the same
 * reference functions as cf_build_block (cosmocore/signal_kernels.py:715-829,
 * cosmocore/basis/pixel.py:802-950) for the mixed path. */
int cf_build_block_planes(int kind, int mode, int na, const double* va, int nb, const double* vb,
                          int lmax, const double* t0, const double* t1, const double* t2,
                          const int* bin_of, void* out, long ld, long row_off, long col_off,
                          long bin_stride, void* outT, long ldT, long rowT_off, long colT_off,
                          long binT_stride, int batch, long tstride, long ostride, int planes,
                          long plane_stride, long planeT_stride, int flags, void* stream);

/* Build-and-reduce: the binned derivative entries of one block (kind, mode,
 * fields and tables as cf_build_block) are consumed where they are formed;
 * nothing but the sums is written:
 *   bias[b]        += scale * sum_{r,c} W[gro + r, gco + c] dC_b[r, c]
 *   q[m * ldq + b] += scale * sum_{r,c} Y[gro + r, m] Y[gco + c, m] dC_b[r, c]
 * over the block and its mirror (scale 1/2 gives 1/2 Tr(W dC_b) and
 * 1/2 y^T dC_b y).  W: symmetric, row stride ldW, or NULL (no bias); Y:
 * nv <= 4 map columns, row stride ldY, or nv = 0; nbins <= 128.  Replaces the
 * dC_b rebuild of qube/spectra.py:1124-1186 (via
 * cosmocore/core.py:1328-1409) together with its traces. */
int cf_build_block_reduce(int kind, int mode, int na, const double* va, int nb, const double* vb, int lmax,
                          const double* t0, const double* t1, const double* t2, const int* bin_of, int nbins,
                          const double* W, long ldW, const double* Y, long ldY, int nv, long gro, long gco,
                          double scale, double* bias, double* q, long ldq, void* stream);

/*
 * C = sum_t A_{ta[t]} B_{tb[t]}^T on tcgen05 (FP32 accumulation in TMEM,
 * partial sums promoted to registers every few k-tiles).  A: planes of
 * M x K (row stride lda, plane stride a_ps), B: planes of N x K.  ta/tb are
 * HOST int arrays of nterms (1..6) plane indices.  Outputs, any may be NULL:
 * X = C as x_planes (1..3) BF16 split planes (M x N, ldx, x_ps); XT = C^T
 * likewise (N x M, ldxt, xt_ps); Cf = C in FP32 (M x N, ldc).  Row strides
 * and plane strides must be multiples of 8 elements, bases 16-byte aligned.
 * Replaces: qube/fisher.py:501-531 (A_b = C^-1 dC_b, matrix_mult) in the
 * mixed path.
 */
int cf_umma_gemm_bf16(int M, int N, int K, int nterms, const int* ta, const int* tb, const void* A,
                      long lda, long a_ps, int a_planes, const void* B, long ldb, long b_ps,
                      int b_planes, void* X, long ldx, long x_ps, int x_planes, void* XT, long ldxt,
                      long xt_ps, float* Cf, long ldc, int* err, void* stream);

/*
 * The product of cf_umma_gemm_bf16 written in FP32 to scattered addresses:
 * element (row, col) goes to Cs[col col_stride + (row / fold) fold_ld +
 * row % fold] (fold = 0: + row) and, when Cs2 is not NULL, to the same
 * offset of Cs2.  With rows = the entries of one block region of the
 * covariance (fold = the region's width, fold_ld = the matrix row stride,
 * Cs at the region's first entry) and columns = parameter points
 * (col_stride = n^2) it writes C(theta) = S(theta) + s N of a batch of points
 * straight into FP32 matrices from the per-multipole basis.
 * Replaces: the per-point covariance build of picslike/picslike.py:301-319
 * (S from cosmocore/signal_kernels.py:164-502 plus the scaled noise) in the
 * mixed likelihood.
 */
int cf_umma_gemm_bf16_scatter(int M, int N, int K, int nterms, const int* ta, const int* tb, const void* A,
                              long lda, long a_ps, int a_planes, const void* B, long ldb, long b_ps, int b_planes,
                              float* Cs, float* Cs2, long col_stride, int fold, long fold_ld, int* err,
                              void* stream);

/*
 * Fisher contraction on tcgen05 with FP64 promotion of the partial sums:
 *   F[(p_off+p) ldF + q_off+q] += scale sum_t sum_{k<K1, l<K2}
 *                                 X_{ta[t]}[p sXp + k ldX + l] Y_{tb[t]}[q sYq + k ldY + l]
 * (and the mirror entry when sym), X/Y BF16 planes x_ps / y_ps apart.  F is
 * FP64 and accumulated with atomics over `splits` CTAs per output tile
 * (splits <= 0 picks a split that fills the GPU); zero it first.
 * Replaces: qube/fisher.py:557-607 and cosmocore/basics/linalg.py:66-98
 * (F_ij = 1/2 Tr(A_i A_j)) in the mixed path.
 */
int cf_umma_trace_bf16(int P1, int P2, int K1, int K2, int nterms, const int* ta, const int* tb,
                       const void* X, long sXp, long ldX, long x_ps, int x_planes, const void* Y,
                       long sYq, long ldY, long y_ps, int y_planes, double scale, double* F, long ldF,
                       long p_off, long q_off, int sym, int splits, int* err, void* stream);

/* cf_umma_trace_bf16 with output row p scattered to F row row_map[p] and
 * column q to F column col_map[q] (device int arrays). */
int cf_umma_trace_bf16_mapped(int P1, int P2, int K1, int K2, int nterms, const int* ta, const int* tb,
                              const void* X, long sXp, long ldX, long x_ps, int x_planes, const void* Y,
                              long sYq, long ldY, long y_ps, int y_planes, double scale, double* F,
                              long ldF, const int* row_map, const int* col_map, int sym, int splits,
                              int* err, void* stream);

/* Bound of every wait of the tcgen05 kernels on a pipeline barrier, in ns
 * (default 2 s; ns < 0 restores it; 0 gives up at the first unsatisfied
 * try).  A wait that runs out aborts the launch cleanly: issued copies and
 * MMAs are drained (with the 2 s bound), TMEM is freed and the launch's error
 * flag is set.  For failure-path tests and watchdogs.  Returns the previous
 * bound.  No counterpart in the reference. */
long long cf_umma_set_wait_limit(long long ns);

/* CF_ERR_TIMEOUT if the device error flag `err` of a tcgen05 launch is set,
 * else CF_OK.  Synchronises `stream`.  No counterpart in the reference. */
int cf_umma_status(const int* err, void* stream);

/* Promotion interval of the tensor-core kernels: k-tiles of 64 summed in one
 * FP32 TMEM accumulator before promotion (1, 2, 4, 8 or 16; default 16).
 * Returns the previous value.  No counterpart in the reference. */
int cf_umma_set_promotion(int kc);

/* Trace contractions (cf_umma_trace_bf16*) on CTA pairs: 256 x 128 output
 * tiles with tcgen05.mma.cta_group::2, each CTA loading its 128 rows of X and
 * 64 of the tile's 128 rows of Y, when both operands carry two or three planes
 * and P1 > 128 (on = 1, the default), or one CTA per 128 x 128 tile (on = 0).
 * Returns the previous setting. */
int cf_umma_set_trace_pairs(int on);

/* Form of cf_umma_gemm_bf16: 1 (default) loads every plane of a 32-wide
 * k-slice into one pipeline stage and keeps the leading product apart from
 * the corrections in a second TMEM accumulator, when both operands carry the
 * same 2 or 3 planes; 2 does the same for three planes of 64-wide k-tiles
 * on CTA pairs (clusters of two CTAs on neighbouring SMs,
 * tcgen05.mma.cta_group::2 on 256-row tiles, each CTA holding half of B,
 * two stages of 96 KB per CTA); 0 walks 64-wide k-tiles term by term.
 * Returns the previous setting.  No counterpart in the reference. */
int cf_umma_set_all_planes(int on);

/* Row tiles per group in the persistent tile order of the tcgen05 kernels
 * (default 16): the CTAs running at one time share group_m A row panels,
 * which stay in L2 while the group's column tiles are swept.  Returns the
 * previous value.  No counterpart in the reference. */
int cf_umma_set_group(int group_m);

/* ---- Mixed-precision pixel likelihood (FP32 factor, FP64-refined chi2) ---- */

/* Bytes of workspace cf_potrf_f32 needs for `batch` problems of order n. */
size_t cf_potrf_f32_workspace(int n, int batch);

/*
 * FP32 GEMM with BF16 split products on the tcgen05 tensor cores:
 *   C_z = alpha A_z B_z^T + beta C_z,  A_z M x K, B_z N x K (K contiguous),
 * each operand split into three BF16 planes and the six plane products with
 * i + j <= 2 accumulated in FP32 (~24 significant bits).  Batch z < batch,
 * element strides sA, sB, sC.  lower_only bit 0 skips output tiles strictly
 * above the diagonal.  info (optional, int[batch]): -3 for a problem whose
 * tile saw a barrier wait run out (then its C is not written).
 * Replaces: the FP32 products of the Cholesky used by the mixed likelihood
 * (picslike/picslike.py:643-664, cosmocore/basics/linalg.py:362-474 in FP64
 * in the reference).
 */
int cf_sgemm_bf16x6(int M, int N, int K, float alpha, const float* A, long lda, long sA, const float* B, long ldb,
                    long sB, float beta, float* C, long ldc, long sC, int batch, int lower_only, int* info,
                    void* stream);

/* Bound of the barrier waits of cf_sgemm_bf16x6 in ns (ns < 0: default 2 s;
 * 0: give up at the first unsatisfied try).  Returns the previous bound.
 * No counterpart in the reference. */
long long cf_sgemm_bf16x6_set_wait_limit(long long ns);

/* Operand stages of cf_sgemm_bf16x6: 1 (default: two CTAs per SM) or 2 (one
 * CTA per SM, double-buffered).  Returns the previous setting.
 * No counterpart in the reference. */
int cf_sgemm_bf16x6_set_stages(int stages);

/* Product kernel of cf_potrf_f32: 1 = cf_sgemm_bf16x6 on the tensor cores
 * (default), 0 = an FP32 SIMT kernel.  Returns the previous setting.
 * No counterpart in the reference. */
int cf_potrf_f32_set_tensor(int on);

/* Panels of 64 columns per pass of cf_potrf_f32 (2 or 4; default 4): the
 * trailing update runs once per pass with K = 64 x panels.  Returns the
 * previous setting.  No counterpart in the reference. */
int cf_potrf_f32_set_group(int panels);

/* Blocked lower Cholesky in FP32, in place (batch), 64-wide panels with FP32
 * GEMM updates; info as for cf_potrf.  The factor of the mixed likelihood:
 * replaces cosmocore/basics/linalg.py:362-406 (cholesky_factor) at FP32. */
int cf_potrf_f32(int n, float* A, long lda, long strideA, int batch, void* work, int* info, void* stream);

/* Z_b = a X_b + c_b W_b in FP64 (Z may be NULL) plus its FP32 copy Z32_b;
 * c_b = cvec[b] if cvec else c.  C = S + s N of picslike/picslike.py:301-319
 * in both precisions. */
int cf_axpby_f32(long count, double a, const double* X, long strideX, double c, const double* cvec,
                 const double* W, long strideW, double* Z, long strideZ, float* Z32, long strideZ32,
                 int batch, void* stream);

/* chi2[b nrhs + m] = 2 |L_b^-1 x|^2 - v^T C_b v, v = (L_b L_b^T)^-1 x: one FP64
 * refinement step on the FP32 factor L_b of the FP64 C_b (lower triangle
 * read), second-order accurate; logdet[b] = 2 sum ln (L_b)_ii.  n <= 12288.
 * Replaces picslike/picslike.py:643-664 and cosmocore/basics/linalg.py:430-474
 * in the mixed likelihood. */
int cf_chi2_logdet_mixed(int n, const float* L, long lda, long strideL, const double* C, long ldc,
                         long strideC, int batch, const double* X, long ldx, long strideX, int nrhs,
                         double* chi2, double* logdet, void* stream);

/* cf_chi2_logdet_mixed with C in FP32 (the matrices the FP32 factor was
 * computed from); the refinement arithmetic stays FP64.  Same replaced
 * reference code. */
int cf_chi2_logdet_mixed_c32(int n, const float* L, long lda, long strideL, const float* C, long ldc,
                             long strideC, int batch, const double* X, long ldx, long strideX, int nrhs,
                             double* chi2, double* logdet, void* stream);

/* The two mixed chi2 forms with the FP32 factor's diagonal-block inverses as
 * cf_potrf_f32 leaves them in its workspace (strideD =
 * cf_potrf_f32_dinv_stride(n) floats between problems): 64-row blocks, each
 * diagonal solve a block-times-vector product.  Same replaced reference code. */
int cf_chi2_logdet_mixed_dinv(int n, const float* L, long lda, long strideL, const float* Dinv, long strideD,
                              const double* C, long ldc, long strideC, int batch, const double* X, long ldx,
                              long strideX, int nrhs, double* chi2, double* logdet, void* stream);
int cf_chi2_logdet_mixed_c32_dinv(int n, const float* L, long lda, long strideL, const float* Dinv,
                                  long strideD, const float* C, long ldc, long strideC, int batch,
                                  const double* X, long ldx, long strideX, int nrhs, double* chi2,
                                  double* logdet, void* stream);

/* Floats between consecutive problems' diagonal-block inverses in the
 * cf_potrf_f32 workspace (it keeps every one).  No counterpart in the
 * reference. */
size_t cf_potrf_f32_dinv_stride(int n);

/* ---- Quadratic forms of many maps ----
 * q[m ldq + p0 + b] += scale sum_{j<J} W[(b rows_per_bin + j) ldW + m] Y[(yoff + j) ldY + m]
 * for b < nb, m < nmaps, with W = D^T Y from one GEMM against the stacked
 * derivative blocks of a spectrum: q_b(m) = 1/2 y_m^T dC_b y_m for every map
 * at once.  Replaces the per-bin loop of qube/spectra.py:1124-1186 for many
 * simulations. */
int cf_qform_reduce_f64(int nb, int J, long rows_per_bin, const double* W, long ldW, const double* Y, long ldY,
                        long yoff, int nmaps, double scale, double* q, long ldq, int p0, void* stream);
int cf_qform_reduce_f32(int nb, int J, long rows_per_bin, const float* W, long ldW, const double* Y, long ldY,
                        long yoff, int nmaps, double scale, double* q, long ldq, int p0, void* stream);

/* ---- Emulator network (BF16 weights, FP32 accumulation) and sampler ----
 * No counterpart in the reference: the MLP emulator of -2 Delta lnL and the
 * delayed-acceptance Metropolis sampler built on the exact likelihood. */

/* out = act(A W^T + b): A M x K FP32 (lda), W N x K BF16, b N FP32 (or NULL),
 * act 1 = SiLU, 0 = linear; Z (pre-activation, may be NULL) and out M x N (ldo). */
int cf_mlp_dense_fwd(int M, int N, int K, const float* A, long lda, const void* W, const float* b,
                     int act, float* Z, float* out, long ldo, void* stream);

/* dZ_prev = (dZ W) * silu'(Z_prev): dZ M x N, W N x K BF16, Z_prev / dZ_prev M x K. */
int cf_mlp_dense_bwd_data(int M, int N, int K, const float* dZ, const void* W, const float* Zprev,
                          float* dZprev, void* stream);

/* dW = dZ^T A_prev (N x K) and db = column sums of dZ (may be NULL). */
int cf_mlp_dense_bwd_weight(int M, int N, int K, const float* dZ, const float* Aprev, long lda, float* dW,
                            float* db, void* stream);

/* Weighted MSE sum w (y - t)^2 / sum w (w may be NULL), gradient dy, loss to *loss. */
int cf_mlp_mse(int M, const float* y, const float* t, const float* w, float* dy, float* loss, void* stream);

/* Adam step over `count` FP32 parameters; *step (device int) is incremented
 * and sets the bias corrections; p16 (may be NULL) receives the BF16 copy. */
int cf_mlp_adam(long count, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                float eps, int* step, void* p16, void* stream);

/* y = bf16(x) for count values. */
int cf_to_bf16(long count, const float* x, void* y, void* stream);

/* Proposal theta_p = theta + Lp xi for chains neither pending nor finished;
 * xin = theta_p mapped from [lo, hi] to [-1, 1]; active 0 idle / 1 inside /
 * 2 outside the box. */
int cf_mcmc_propose(int C, int D, const double* theta, const int* pending, const int* steps, int max_steps,
                    const double* Lp, const double* xi, const double* lo, const double* hi, double* theta_p,
                    float* xin, int* active, void* stream);

/* Delayed-acceptance stage 1 (emulator: lnL~ = -(mu + sigma y) / 2). */
int cf_mcmc_stage1(int C, int D, const int* active, const float* y, double mu, double sigma, const double* u,
                   const double* theta, double* ltil, double* ltil_p, int* pending, int* steps,
                   double* samples, int max_steps, int* n_stage1, void* stream);

/* Delayed-acceptance stage 2 (exact lnL of the pending proposals). */
int cf_mcmc_stage2(int C, int D, const double* lexact_p, double* lexact, double* ltil, const double* ltil_p,
                   const double* u, double* theta, const double* theta_p, int* pending, int* steps,
                   double* samples, int max_steps, int* n_exact, int* n_accept, void* stream);

/* Plain exact-likelihood Metropolis acceptance. */
int cf_mcmc_mh_accept(int C, int D, const int* active, const double* lexact_p, double* lexact, const double* u,
                      double* theta, const double* theta_p, int* steps, double* samples, int max_steps,
                      int* n_exact, int* n_accept, void* stream);

/* Two-level delayed acceptance, emulator sub-chain step: chains with
 * active == 1 move theta_s to theta_p with probability
 * min(1, exp(lnL~(theta_p) - ltil_s)) (lnL~ = -(mu + sigma y) / 2). */
int cf_mcmc_sub_accept(int C, int D, const int* active, const float* y, double mu, double sigma, const double* u,
                       const double* theta_p, double* theta_s, double* ltil_s, int* n_sub_accept, void* stream);

/* Two-level delayed acceptance, exact stage: the sub-chain end point theta_s
 * (exact lnL lexact_p) replaces theta with probability
 * min(1, exp([lexact_p - lexact] - [ltil_s - ltil])); unfinished chains
 * record a step; theta_s / ltil_s are reset to the chain's point. */
int cf_mcmc_sub_final(int C, int D, const double* lexact_p, double* lexact, double* ltil, double* ltil_s,
                      const double* u, double* theta, double* theta_s, int* steps, double* samples, int max_steps,
                      int* n_exact, int* n_accept, void* stream);

/* Fused emulator sub-chains: one CTA per chain computes lnL~ at theta (into
 * ltil) and runs J Metropolis steps on the emulator posterior (proposals
 * Lp xi[j][c], uniforms u[j][c]; xi J x C x D, u J x C), end point into
 * theta_s / ltil_s, accepted moves added to n_sub.  The emulator: flat
 * parameter vector (per layer W out x in row-major, then b) read as BF16
 * weights (w16, 16-byte aligned) and FP32 biases (w32); sizes
 * D -> 256 x n_hidden -> 1, SiLU, lnL~ = -(mu + sigma y) / 2.  Chains with
 * steps >= max_steps copy theta to theta_s. */
int cf_mcmc_subchain(int C, int D, int J, int n_hidden, const double* theta, const int* steps, int max_steps,
                     const double* Lp, const double* xi, const double* u, const double* lo, const double* hi,
                     const void* w16, const float* w32, double mu, double sigma, double* theta_s, double* ltil,
                     double* ltil_s, int* n_sub, void* stream);

/* ---- harmonic basis (basis="harmonic") ----------------------------------
 * V: real spherical harmonics of the active pixels, rows component-major
 * (T of a spin-0 field; E then B of a spin-2 field over its [Q | U] columns),
 * then multipole l in [lmin, lmax], then m = 0 and (cos m, sin m) pairs.
 * dC/dC_l = t_l V_(u,l)^T V_(v,l) (+ transpose for cross spectra) turns the
 * Fisher traces, the noise bias and the quadratic forms into contractions of
 * G = V C^-1 V^T, Z N Z^T and z = Z x (Z = V C^-1).
 * Replaces: cosmocore/basis/harmonic_basis.py:20-180 (V, with
 * cosmocore/basics/legendre.py:153-210 and cosmocore/basics/wigner.py:12-120),
 * the harmonic Fisher of qube/fisher.py:416-500, 575-583 and the harmonic
 * quadratic forms of cosmocore/basis/harmonic.py:191-1252. */

/* Rows [row0, row0 + (lmax+1)^2 - lmin^2) of V (row stride ldV, zeroed by the
 * caller) for one component over columns col0..: spin 0, or spin 2 with
 * is_b 0 (E) / 1 (B) over [Q | U] (2 npix columns).  vec: SoA x[npix] y[npix]
 * z[npix].  lmax <= 255; spin 2 needs lmin >= 2. */
int cf_harmonic_operator(int spin, int is_b, int npix, const double* vec, int lmin, int lmax, double* V, long ldV,
                         long row0, long col0, void* stream);

/* LV[(u,l,m), j] = sum_v lam[(u nc + v) Lp + l] V[(v,l,m), j] for nm rows and
 * ncol columns; rowinfo int[2 nm] (component, multipole) of each row; off
 * long[nc Lp] first row of (component, multipole). */
int cf_harmonic_lambda(long nm, long ncol, int nc, int lmin, const int* rowinfo, const long* off, const double* lam,
                       int Lp, const double* V, long ldV, double* LV, long ldL, void* stream);

/* F += the binned Fisher matrix (nspec nb square, row stride ldF) from
 * G = V C^-1 V^T (row stride ldG); nc <= 3 components; su / sv int[nspec]
 * the components of each spectrum; tab / bin [nspec Lp] the weight and bin of
 * each multipole (bin -1 outside the bins). */
int cf_harmonic_fisher(int nc, int lmin, int lmax, int Lp, const double* G, long ldG, const long* off, int nspec,
                       const int* su, const int* sv, const double* tab, const int* bin, int nb, double* F, long ldF,
                       void* stream);

/* out[p] (per_col 0) or out[k ldo + p] (per_col 1) += 1/2 t_(s,l) sum_m
 * A_(u,l,m) . B_(v,l,m) (+ the swapped pair for cross spectra), summed over
 * the ncol columns or per column: A = Z N, B = Z gives the raw noise bias,
 * A = B = Z X the raw quadratic forms. */
int cf_harmonic_pair(int lmin, int lmax, int Lp, const double* A, long ldA, const double* B, long ldB, long ncol,
                     int per_col, const long* off, int nspec, const int* su, const int* sv, const double* tab,
                     const int* bin, int nb, double* out, long ldo, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CFB200_H */
