/*
 * vbcsr_b200 — C ABI of the B200 (sm_100a) variable-block sparse engine.
 *
 * This is the drop-in boundary beneath the `vbcsr_core` Python extension: the
 * C++ host core (graph, host mirrors, Python buffers) calls only the functions
 * below, and any other host language can bind them directly (plain pointers,
 * sizes and an opaque stream; no C++ or torch types cross it).
 *
 * Conventions
 *  - Every function returns 0 on success and a negative VBG_E* code on error;
 *    vbg_last_error() returns a message for the calling thread.  Nothing
 *    throws across the ABI.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *    stream).  Functions suffixed _host take HOST buffers and synchronise the
 *    stream before returning; all others take DEVICE pointers and are
 *    asynchronous with respect to the host.
 *  - Values are stored exactly like the reference's BlockSpMat export
 *    (vbcsr/core/block_csr.hpp:1202-1248 get_values): blocks in slot order
 *    (row by row, columns ascending inside a row), each block row-major r x c.
 *    Complex values are interleaved (re, im) doubles.
 *  - A multivector is row-major with a padded leading dimension `ld` and zero
 *    pad lanes, the reference's DistMultiVector layout
 *    (vbcsr/core/dist_multivector.hpp:24-47): element (row, vec) at
 *    data[row * ld + vec].  A plain vector is the k = 1, ld = 1 case.
 */
#ifndef VBCSR_B200_H
#define VBCSR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VBG_OK 0
#define VBG_E_ARG (-1)     /* invalid argument (null, size, mismatch) */
#define VBG_E_CUDA (-2)    /* CUDA runtime error */
#define VBG_E_NOMEM (-3)   /* device allocation failed */
#define VBG_E_STATE (-4)   /* operation not valid for this handle */
#define VBG_E_DEVICE (-5)  /* device-side check failed (bounded wait / overflow) */

/* Scalar types.  F64 and C128 are the reference's BlockSpMat_Double and
 * BlockSpMat_Complex (vbcsr/pybind_vbcsr.cpp:476-479). */
#define VBG_F64 0
#define VBG_C128 1

/* Matrix kinds, same names as the reference (vbcsr/core/block_csr.hpp:33-50,
 * detection at :2771-2798): every block 1x1 -> CSR, all equal -> BSR,
 * else VBCSR.  All three run on the same variable-block kernels here. */
#define VBG_KIND_CSR 0
#define VBG_KIND_BSR 1
#define VBG_KIND_VBCSR 2

/* Precision of the bulk Chebyshev/KPM arithmetic. */
#define VBG_PREC_F64 0 /* plain FP64: the drop-in path */
#define VBG_PREC_F32 1 /* FP32 values and vectors, FP32 accumulation, FP64 moment sums */

typedef struct vbg_matrix vbg_matrix;

int vbg_version(void);
const char* vbg_last_error(void);
/* Number of visible CUDA devices (0 when none); never fails. */
int vbg_device_count(void);
/* Device-side status of the current device's kernels since the last clear
 * (no counterpart in the reference): bit 0 = a pipelined multivector apply
 * gave up waiting for staged data (its results are then wrong).  Synchronises
 * the device; `clear` != 0 resets the word. */
#define VBG_STATUS_STAGE_TIMEOUT 1u
int vbg_device_status(unsigned* status, int clear);
/* Process-wide library options (no counterpart in the reference).
 *   "apply.chain"  multivector applies that run on the tiled kernel use its
 *                  chained variant (VBG_KERNEL_CHAIN) when a chain plan fits
 *                  the matrix: 1 always, 0 never (the unchained tiles),
 *                  2 (default) as the autotuner decides.
 *   "apply.autotune" 1 (default): the first forward multivector apply with a
 *                  given leading dimension and precision on a matrix (outside
 *                  stream capture; vbg_kpm_moments* before their capture)
 *                  times the kernels that can run it -- chained tiles, tiles,
 *                  pipelined -- and keeps the fastest for that matrix; the
 *                  trials overwrite Y and the dots, never the accumulator.
 *                  0: the default order (chained tiles for FP32 only).
 *                  vbg_apply_kernel reports the tuned choice once made.
 * An unknown name returns VBG_E_ARG.  Graphs captured before a change keep
 * the kernels they captured. */
int vbg_set_option(const char* name, long long value);
int vbg_get_option(const char* name, long long* value);
/* Device memory of the library (no counterpart in the reference: the
 * reference's matrices live in host memory).  Buffers of 4 MiB and more are
 * cudaMalloc blocks (powers of two from 32 MiB) that the library caches once
 * released; smaller ones come from a stream-ordered pool per device that
 * keeps released memory mapped (up to an eighth of the device memory).
 * vbg_memory_reserve maps `bytes` into the current device's pool ahead of
 * use; vbg_memory_trim returns the cached blocks and the pool's unused memory
 * to the driver.  Both synchronise the device. */
int vbg_memory_reserve(size_t bytes);
int vbg_memory_trim(void);

/* ---------------------------------------------------------------- matrices */

/* Create a square block matrix on the current device from host arrays.
 * Replaces DistGraph::construct_serial + BlockSpMat add_block/assemble
 * (vbcsr/core/dist_graph.hpp:167-312; vbcsr/core/block_csr.hpp:613,861) for
 * the serial case: block_sizes[n_block_rows]; row_ptr[n+1]; col_ind[nnzb]
 * global block columns.  Columns inside a row need not be sorted: they are
 * sorted here (the reference sorts each row's columns, dist_graph.hpp:299);
 * `values`, if not NULL, must already follow the SORTED slot order. */
int vbg_matrix_create(vbg_matrix** out, int dtype, int n_block_rows, const int* block_sizes,
                      const int* row_ptr, const int* col_ind, const void* values, void* stream);
/* The same from a structure already in device memory: row_ptr_dev[n+1] and
 * col_ind_dev[nnzb] are DEVICE arrays (columns ascending within each row:
 * this constructor does not sort; repeated columns are allowed),
 * values_dev (DEVICE, may be NULL = zeros) in slot order; block_sizes[n]
 * is a HOST array.  The structure is checked on the device before use
 * (row pointers, column range, order: VBG_E_ARG on a violation) and the
 * slot offsets, gather records and diagonal slots are built there; the host
 * does O(n) work from the block sizes.  For structures generated on the GPU
 * (the reference builds them on the host: dist_graph.hpp:167-312). */
int vbg_matrix_create_device(vbg_matrix** out, int dtype, int n_block_rows, const int* block_sizes, int64_t nnzb,
                             const int* row_ptr_dev, const int* col_ind_dev, const void* values_dev,
                             void* stream);
int vbg_matrix_destroy(vbg_matrix* m);
/* Deep copy (vbcsr/core/block_csr.hpp:579 duplicate). */
int vbg_matrix_duplicate(const vbg_matrix* m, vbg_matrix** out, void* stream);
int vbg_matrix_info(const vbg_matrix* m, int* dtype, int* n_block_rows, int64_t* nnzb,
                    int64_t* nnz, int64_t* n_scalar_rows, int* kind);
/* Host copies of the structure: row_ptr[n+1], col_ind[nnzb], block_sizes[n]. */
int vbg_matrix_get_structure(const vbg_matrix* m, int* row_ptr, int* col_ind, int* block_sizes);
/* Host copy of all values in slot order (block_csr.hpp:1202 get_values). */
int vbg_matrix_get_values(const vbg_matrix* m, void* values, void* stream);
int vbg_matrix_set_values(vbg_matrix* m, const void* values, void* stream);
/* Same from device memory (stream-ordered; no host synchronisation). */
int vbg_matrix_set_values_device(vbg_matrix* m, const void* values_dev, void* stream);
/* Device pointer to the FP64/C128 values (slot order) and to the value
 * offset of each slot (int64, nnzb+1 entries).  Read-only for callers: the
 * library keeps derived copies of the values (FP32, kernel layout) that a
 * write through this pointer would leave stale; change values with
 * vbg_matrix_set_values or the vbg_matrix_* operations. */
int vbg_matrix_device_values(const vbg_matrix* m, void** values, const int64_t** slot_offsets);
/* Block Frobenius norms in slot order into device memory
 * (vbcsr/core/block_csr.hpp:2487 compute_block_norms). */
int vbg_matrix_block_norms(const vbg_matrix* m, double* norms_dev, void* stream);

/* ------------------------------------------------- apply (SpMV / SpMM) */

/* y = A x.  block_csr.hpp:985 mult -> detail/kernels/vbcsr_apply.hpp:193-275. */
int vbg_spmv(const vbg_matrix* m, const void* x, void* y, void* stream);
/* y = A^H x.  block_csr.hpp:1024 mult_adjoint -> vbcsr_apply.hpp:57-74,342-424. */
int vbg_spmv_adjoint(const vbg_matrix* m, const void* x, void* y, void* stream);
/* Y = A X, X/Y row-major with leading dimension ld >= k (pad lanes zero).
 * block_csr.hpp:1011 mult_dense -> vbcsr_apply.hpp:277-340. */
int vbg_spmm(const vbg_matrix* m, int k, int ld, const void* X, void* Y, void* stream);
/* The forward kernel an apply (vbg_spmv / vbg_spmm / vbg_cheb_step) with
 * leading dimension ld and `precision` (VBG_PREC_*) runs on this matrix, for
 * 16-byte-aligned buffers (no counterpart in the reference).  Builds the
 * value layout and tile plan that choice needs, as the first apply would. */
#define VBG_KERNEL_VECTOR 0 /* ld == 1: a warp per block row, lanes over (block, row) pairs */
#define VBG_KERNEL_ROWS 1   /* a warp per block row, X rows read per lane */
#define VBG_KERNEL_PIPE 2   /* a warp per block row, spans staged by bulk copies */
#define VBG_KERNEL_TILE 3   /* a CTA per tile of block rows, X ranges staged once per tile */
#define VBG_KERNEL_CHAIN 4  /* tiles chained per persistent CTA, X rows cached across tiles */
#define VBG_KERNEL_SCALAR_ROWS 5 /* ld == 1: 1-8 threads per scalar row, the row's blocks split among them */
int vbg_apply_kernel(const vbg_matrix* m, int ld, int precision, int* kernel);
/* Block rows per tile of the tiled kernel's plan for applies at this leading
 * dimension and precision (no counterpart in the reference): the height the
 * autotuner kept (it times tiles of at most 16, 12 and 8 block rows), or the
 * tallest that fits before it has run; 0 when no tile plan exists yet. */
int vbg_apply_tile_rows(const vbg_matrix* m, int ld, int precision, int* rows);
/* Y = A^H X.  block_csr.hpp:1038 mult_dense_adjoint. */
int vbg_spmm_adjoint(const vbg_matrix* m, int k, int ld, const void* X, void* Y, void* stream);
/* Host-buffer variants (copies in and out inside the call, stream synchronised). */
int vbg_spmv_host(const vbg_matrix* m, const void* x, void* y, void* stream);
int vbg_spmm_host(const vbg_matrix* m, int k, const void* X, void* Y, void* stream);

/* ------------------------------------------------ fused Chebyshev step */

/* One step of the Chebyshev three-term recurrence, fused with its moment dot
 * products (the loop bodies of examples/ex08_graphene_dos.py:109-114,
 * examples/inp_nanocrystal_dos/kpm.py:40-74 and vbcsr/utils.py:71-126):
 *
 *     Y = alpha * (A X) + beta * X + gamma * Xprev
 *
 * Xprev may be NULL when gamma == 0.  If dots != NULL the kernel also writes
 *     dots[0] = sum over all k columns of Re <Xdot, Y>   (Xdot = X if dot_with
 *               is NULL, else dot_with)
 *     dots[1] = sum over all k columns of <Y, Y>
 * to DEVICE memory, reduced in a fixed order (deterministic).  If acc != NULL
 * it also updates acc += acc_coef * Y (acc_coef complex for C128: re, im).
 * k, ld as for vbg_spmm; ld == 1 with k == 1 is a plain vector. */
int vbg_cheb_step(const vbg_matrix* m, int k, int ld, double alpha, double beta, double gamma,
                  const void* X, const void* Xprev, void* Y, const void* dot_with, double* dots,
                  void* acc, double acc_coef_re, double acc_coef_im, void* stream);
/* vbg_cheb_step with the adjoint: Y = alpha (A^H X) + beta X + gamma Xprev,
 * acc += (cre + i cim) Y, dots as vbg_cheb_step.  One step of the adjoint
 * Chebyshev recurrence a_n = s_n + w H~^H a_{n+1} - a_{n+2} of a gradient
 * through a Chebyshev series (acc = s_n, alpha = w / scale, beta =
 * -w center / scale, gamma = -1); none in the reference, which has no
 * gradients. */
int vbg_cheb_step_adjoint(const vbg_matrix* m, int k, int ld, double alpha, double beta, double gamma, const void* X,
                          const void* Xprev, void* Y, const void* dot_with, double* dots, void* acc, double cre,
                          double cim, void* stream);

/* A whole Chebyshev series in one call (the reference's Python loop of
 * examples/ex09_graphene_dynamics.py:102-133, vbcsr/utils.py:71-126):
 * psi = sum_{n<M} c_n t_n with t_0 = V, t_1 = H~ V, t_{n+1} = 2 H~ t_n - t_{n-1}
 * and H~ = (H - center) / scale; c is a HOST array of M complex
 * coefficients (re, im) (imaginary parts ignored for real matrices).  V and
 * psi are N x ld multivectors (psi is written).  With K > 0 the pairs
 * (t_n, t_{n-1}) of n = K, 2K, ... < M are copied to ckpt, pair j = n/K - 1
 * at vectors 2j and 2j + 1 (ckpt holds 2 floor((M - 1) / K) multivectors of
 * N x ld): the checkpoints an adjoint recurrence restarts from.  Each step
 * is one fused apply; the three working vectors are the library's. */
int vbg_cheb_series(const vbg_matrix* m, int k, int ld, const void* V, int M, const double* coeffs, double scale,
                    double center, void* psi, int K, void* ckpt, void* stream);

/* vbg_cheb_step with dots, for callers that cannot let the library allocate
 * device memory (no counterpart in the reference).  vbg_cheb_step allocates
 * its per-CTA reduction scratch on first use; this variant allocates nothing
 * and instead reduces through a fixed array inside the library image (64 KiB
 * of partial sums for at most 4096 thread blocks, plus a counter), held by
 * every GPU that loads the library until the process exits.  Callers that
 * manage all device memory through their own pool, or that must not
 * synchronise the device mid-call, use it.  `dots` is required.  A launch
 * that would need more than 4096 blocks' partials is rejected (VBG_E_ARG)
 * before anything is launched.  The call builds no derived layout: on a
 * matrix that no earlier multivector apply has prepared it runs the
 * row-per-warp kernel (same results within rounding).  The first call on
 * each device looks up the array's device address; under lazy module
 * loading that lookup may load the library's device code on the device
 * (which allocates and synchronises), so make a first call during set-up,
 * before any stream capture or allocation-free section.  All calls share the
 * one array: calls whose kernels overlap on the GPU race on it and must be
 * serialised (e.g. issued on one stream). */
int vbg_cheb_step_noalloc(const vbg_matrix* m, int k, int ld, double alpha, double beta, double gamma,
                          const void* X, const void* Xprev, void* Y, const void* dot_with, double* dots,
                          void* acc, double acc_coef_re, double acc_coef_im, void* stream);

/* KPM moments of A (already rescaled into [-1, 1]) for R random vectors V0
 * (device, row-major with leading dimension ld), all recurrence work on the
 * device.  moments[n] = sum_r Re <v0_r | T_n(A) | v0_r>, n < M (unnormalised,
 * the quantity examples/ex08_graphene_dos.py:99-114 accumulates before
 * dividing by R*N).
 *   precision : VBG_PREC_F64 or VBG_PREC_F32 (FP32 bulk, FP64 sums)
 *   two_moment: 1 = two moments per SpMM (mu_2n = 2<t_n,t_n> - mu_0,
 *               mu_2n+1 = 2<t_n+1,t_n> - mu_1; kpm.py:40-74), 0 = plain
 *               recurrence mu_n = <v0, t_n> (ex08)
 *   use_graph : capture the step loop in a CUDA graph (replayed on later
 *               calls with the same arguments)
 * moments: DEVICE array of M doubles. */
int vbg_kpm_moments(const vbg_matrix* m, int R, int ld, const void* V0, int M, int precision,
                    int two_moment, int use_graph, double* moments, void* stream);
/* Same with HOST V0 (dense row-major N x R) and HOST moments. */
int vbg_kpm_moments_host(const vbg_matrix* m, int R, const double* V0, int M, int precision,
                         int two_moment, double* moments, void* stream);

/* ----------------------------------------------- multivector operations */
/* All on DEVICE buffers of n_rows x ld (k live columns).  Scalars are
 * (re, im); the imaginary part is ignored for F64.
 * vbcsr/core/dist_multivector.hpp:179-206 scale/axpy/axpby, :283-314 bdot. */
int vbg_mv_scale(int dtype, int64_t n_rows, int k, int ld, double re, double im, void* X, void* stream);
/* Y = alpha X + beta Y */
int vbg_mv_axpby(int dtype, int64_t n_rows, int k, int ld, double a_re, double a_im, const void* X,
                 double b_re, double b_im, void* Y, void* stream);
/* out[c] = sum_rows conj(X[row, c]) * Y[row, c], c < k; out is DEVICE, k scalars. */
int vbg_mv_bdot(int dtype, int64_t n_rows, int k, int ld, const void* X, const void* Y, void* out,
                void* stream);
/* X *= Y elementwise (same shape) or, if y_is_vector, X[row, :] *= y[row]. */
int vbg_mv_pointwise(int dtype, int64_t n_rows, int k, int ld, const void* Y, int y_is_vector,
                     void* X, void* stream);
/* Counter-based random fill, vbcsr/core/random_vectors.hpp:52-160 and
 * dist_multivector.hpp:335-373: entry (block b, row-in-block t, column c) is
 * a hash of (seed, global block id, t, c); Rademacher for F64, random phase
 * for C128; normalize scales by 1/sqrt(N). */
int vbg_mv_set_random(const vbg_matrix* m, int k, int ld, uint64_t seed, int normalize, void* X,
                      void* stream);

/* --------------------------------------------- matrix algebra on device */

/* A *= alpha (block_csr.hpp:1053). */
int vbg_matrix_scale(vbg_matrix* m, double re, double im, void* stream);
/* A_ii += alpha on every diagonal block's diagonal (block_csr.hpp:1289). */
int vbg_matrix_shift(vbg_matrix* m, double re, double im, void* stream);
/* A_ii += v_i (block_csr.hpp:1329 add_diagonal); v is a DEVICE vector. */
int vbg_matrix_add_diagonal(vbg_matrix* m, const void* v, void* stream);
/* Trace of A (sum of the diagonal blocks' diagonals) into DEVICE out[0..1]
 * (real, imaginary part), and the Frobenius norm sqrt(sum |a|^2) into DEVICE
 * out[0]: FP64, reduced in a fixed order on the device (no counterpart as
 * one call in the reference; its McWeeny loop, README.md:22-33, leaves
 * these to host numpy).  They use the matrix's reduction scratch, shared
 * with the fused Chebyshev step's dots: calls on one matrix from different
 * streams must be ordered. */
int vbg_matrix_trace(const vbg_matrix* m, double* out, void* stream);
int vbg_matrix_norm_fro(const vbg_matrix* m, double* out, void* stream);
/* Y <- alpha X + beta Y (ops/axpby.hpp:254 VBCSRAxpbyExecutor::run).  When
 * the patterns differ, Y's structure becomes the union pattern. */
int vbg_matrix_axpby(vbg_matrix* Y, double a_re, double a_im, const vbg_matrix* X, double b_re,
                     double b_im, void* stream);
/* Drop blocks with Frobenius norm < threshold (keep >=), threshold <= 0 is a
 * no-op (block_csr.hpp:1399-1528). */
int vbg_matrix_filter_blocks(vbg_matrix* m, double threshold, void* stream);
/* Conjugate transpose A^H as a new matrix (ops/transpose.hpp:179). */
int vbg_matrix_transpose(const vbg_matrix* m, vbg_matrix** out, void* stream);
/* Elementwise conjugate in place (block_csr.hpp:1070). */
int vbg_matrix_conjugate(vbg_matrix* m, void* stream);

/* Thresholded SpGEMM C = A B (block_csr.hpp:1530 spmm ->
 * detail/ops/spmm/vbcsr.hpp:70-115): symbolic keep rule
 * sum_k |A_ik||B_kj| > threshold (ops/spmm/common.hpp:508-735), numeric
 * per-pair skip |A_ik||B_kj| < threshold / nnzblk(A row i)
 * (vbcsr.hpp:372,386), then the Frobenius filter (keep >= threshold) fused
 * into the write-out.  stats (optional, host, 4 entries): symbolic blocks,
 * final blocks, block products executed, scalar flops. */
int vbg_spgemm(const vbg_matrix* A, const vbg_matrix* B, double threshold, vbg_matrix** C,
               int64_t* stats, void* stream);
/* C = A B for a product the caller knows to be Hermitian
 * (BlockSpMat::spmm_hermitian, block_csr.hpp:1597-1617): only the upper
 * block triangle is multiplied (the symbolic phase skips block columns below
 * the row, common.hpp:502-506), with vbg_spgemm's threshold rules; the strict
 * lower triangle is the conjugate transpose of the strict upper one
 * (ops/transpose.hpp:139-198) and every diagonal block is Hermitized
 * ((D + D^H) / 2, block_csr.hpp:1941-1966), so C is exactly Hermitian --
 * and wrong if the true product is not.  About half the block products of
 * vbg_spgemm.  stats: U's symbolic blocks, C's blocks, U's block products,
 * U's scalar flops. */
int vbg_spgemm_hermitian(const vbg_matrix* A, const vbg_matrix* B, double threshold, vbg_matrix** C,
                         int64_t* stats, void* stream);
/* vbg_spgemm (hermitian = 0) or vbg_spgemm_hermitian (hermitian = 1) with
 * the numeric phase's arithmetic in `precision`: VBG_PREC_F32 (real
 * matrices) multiplies the operands' FP32 copies with FP32 accumulation and
 * stores the rounded results in C's FP64 values; block norms, the pair skip
 * and the filter stay FP64.  For the FP32 bulk iterations of McWeeny
 * purification (no counterpart in the reference, which is FP64 only). */
int vbg_spgemm_ex(const vbg_matrix* A, const vbg_matrix* B, double threshold, int precision, int hermitian,
                  vbg_matrix** C, int64_t* stats, void* stream);

/* Fused triple products, upper block triangle only (complete with
 * vbg_matrix_complete_hermitian), with the reference's per-row pair gates
 * and ONE drop of the finished blocks (Frobenius norm < threshold):
 *   vbg_square_polynomial_upper  C = c2 A^2 + c1 A + c0 I, A Hermitian
 *     (BlockSpMat::square_polynomial_upper, block_csr.hpp:1804 ->
 *     ops/spmm/square_polynomial.hpp): pairs (i,k)(k,j) skipped when
 *     |A_ik||A_kj| < threshold / max(1, nnzb(A row i)) (0 for an all-zero
 *     A); A's own columns and the diagonal always reached; coefficients
 *     complex as (re, im), the imaginary parts ignored for real matrices;
 *   vbg_rarh_upper  C = A B A^H, A and B Hermitian (BlockSpMat::rarh_upper,
 *     block_csr.hpp:1825 -> ops/spmm/rarh.hpp);
 *   vbg_rhar_upper  C = A^H B A, B Hermitian (BlockSpMat::rhar_upper,
 *     block_csr.hpp:1849 -> ops/spmm/rhar.hpp):
 *     stage one T = L B (L = A, or A^H) skips a pair when |L_ik||B_kl| <
 *     threshold / (2 max(1, nnzb(L row i)) nnzb(B row k) max|A|), stage two
 *     C = T A when bound(T_il)|A_lj| < threshold / (2 nnzb(T row i)), with
 *     bound(T_il) the sum of the norms of T_il's pairs.
 * Unlike the reference, which holds one intermediate row per thread, the
 * intermediate T (or A^2) is formed in device memory; the gates, and so the
 * result, are the same. */
int vbg_square_polynomial_upper(const vbg_matrix* A, double c2_re, double c2_im, double c1_re, double c1_im,
                                double c0_re, double c0_im, double threshold, vbg_matrix** C, void* stream);
int vbg_rarh_upper(const vbg_matrix* A, const vbg_matrix* B, double threshold, vbg_matrix** C, void* stream);
int vbg_rhar_upper(const vbg_matrix* A, const vbg_matrix* B, double threshold, vbg_matrix** C, void* stream);
/* Completes an upper-block-triangular m in place: the strict lower triangle
 * becomes the conjugate transpose of the strict upper one and every diagonal
 * block is Hermitized, (D + D^H) / 2 (BlockSpMat::complete_hermitian,
 * block_csr.hpp:1909-1915, hermitize_diagonal_blocks :1943-1969). */
int vbg_matrix_complete_hermitian(vbg_matrix* m, void* stream);

/* Batched KPM moments of independent Hamiltonians in one recurrence: m is
 * block diagonal, segment s spanning block rows [seg_rows[s], seg_rows[s+1])
 * (HOST array, nseg + 1 entries, seg_rows[nseg] = n); V0 holds each
 * Hamiltonian's R >= 2 random vectors in its rows.  Every Chebyshev step is
 * one apply over all segments (rows of all Hamiltonians interleave in the
 * grid, no per-matrix launches) whose per-row moment dots are summed per
 * segment.  moments: DEVICE nseg x M, row s = the moments of segment s, as
 * vbg_kpm_moments (the batched loop of examples/inp_nanocrystal_dos/kpm.py:40-74
 * run for many matrices at once; no counterpart as one call in the
 * reference). */
int vbg_kpm_moments_batched(const vbg_matrix* m, int nseg, const int* seg_rows, int R, int ld, const void* V0,
                            int M, int precision, int two_moment, int use_graph, double* moments, void* stream);

/* ------------------------------------------------------------- gradients */

/* Pattern-restricted outer products (SDDMM), the matrix term of the
 * backward of Y = A X (no counterpart in the reference, which has no
 * gradients): for every stored block (i, j) of A
 *     out_ij += alpha * G_i X_j^H
 * where G_i are the r rows of G at block row i and X_j the c rows of X at
 * block column j, k columns each (multivectors with leading dimension ld,
 * ld = k = 1 for vectors).  `out` is a DEVICE array with A's value layout
 * (slot order, row-major blocks).  For a real loss with dL/dY* = G this adds
 * dL/dA* on A's pattern. */
int vbg_sddmm(const vbg_matrix* m, int k, int ld, const void* G, const void* X, double alpha_re,
              double alpha_im, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VBCSR_B200_H */
