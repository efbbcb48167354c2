/* trl_cuda.h — C ABI of the B200 (sm_100a) backend for trl's block Lanczos eigensolver.
 *
 * This is the drop-in boundary. The C++20 backend in include/trl/impl/cuda/ (namespace
 * trl::cuda) implements trl's backend concepts (include/trl/concepts.hh:26-188 in the
 * reference) by calling these functions; the reference's Lanczos driver
 * (include/trl/eigensolvers/lanczos.hh) is used unchanged on top of it.
 *
 * Conventions
 *  - Every function returns an int status (TRL_OK = 0). No C++ exception crosses the ABI.
 *  - All vector/matrix pointers are DEVICE pointers owned by the caller unless a parameter
 *    name says host_. Work is enqueued on the handle's stream and is asynchronous unless
 *    stated otherwise.
 *  - A "block vector" of block size bs is an n x bs row-major slab; a multivector is a
 *    sequence of such slabs with stride n*bs elements (the reference layout,
 *    impl/openmp/multivector.hh:88). A "block matrix" is a grid of bs x bs row-major blocks
 *    stored block-row-major, block (i,j) at (i*block_cols + j)*bs*bs
 *    (impl/openmp/blockmatrix.hh:56-57). Block-matrix entries are always FP64.
 *  - dtype selects the element type of block vectors and CSR values: TRL_F64 or TRL_F32.
 *    FP32 data are widened to FP64 for every product; dots/Grams accumulate in FP64.
 *  - Supported block sizes: 1, 2, 4, 8, 16.
 *  - A handle is not thread-safe; use one handle per host thread / stream.
 *  - Numerical breakdown found on the device (a Cholesky pivot <= 0) does not stop the
 *    stream: it is recorded in the handle's device status word and reported by the next
 *    trl_cuda_synchronize() / trl_cuda_small_eigen() as TRL_ECHOLESKY.
 */
#ifndef TRL_CUDA_H
#define TRL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct trl_cuda_context* trl_cuda_handle;

enum trl_status {
  TRL_OK = 0,
  TRL_EINVAL = 1,     /* invalid argument (size, block size, null pointer, alignment) */
  TRL_ENOMEM = 2,     /* device allocation failed */
  TRL_ECUDA = 3,      /* CUDA runtime / launch error */
  TRL_ECHOLESKY = 4,  /* Cholesky pivot <= 0 in orthonormalize (evp_base.hh:55) */
  TRL_EEIGEN = 5,     /* projected eigensolver failed (evp_base.hh:96) */
  TRL_ETIMEOUT = 6,   /* a bounded device-side wait gave up */
  TRL_ENOTSUP = 7     /* unsupported combination (block size, dtype) */
};

enum trl_dtype { TRL_F64 = 0, TRL_F32 = 1 };

enum trl_copy_kind { TRL_H2D = 0, TRL_D2H = 1, TRL_D2D = 2 };

/* CSR operator, full storage (both triangles), int32 indices
 * (examples/sycl/csrevp.hh:16-23 in the reference). values has value_dtype. */
typedef struct trl_csr {
  int64_t n;
  int64_t nnz;
  const int32_t* rowptr; /* n+1 */
  const int32_t* colind; /* nnz, sorted within each row */
  const void* values;    /* nnz */
  int value_dtype;       /* TRL_F64 or TRL_F32 */
} trl_csr;

/* ---- context --------------------------------------------------------------------- */

/* Creates a handle on `device`. stream: a cudaStream_t to enqueue on, or NULL to create a
 * private non-blocking stream owned by the handle. The legacy default stream (whose
 * cudaStream_t value is 0) is selected with cudaStreamLegacy, i.e. (void*)1. */
int trl_cuda_create(trl_cuda_handle* handle, int device, void* stream);
int trl_cuda_destroy(trl_cuda_handle handle);
/* Waits for the handle's stream; returns and clears any recorded device-side status. */
int trl_cuda_synchronize(trl_cuda_handle handle);
void* trl_cuda_stream(trl_cuda_handle handle);
const char* trl_cuda_last_error(trl_cuda_handle handle);
const char* trl_cuda_status_string(int status);
/* Number of kernels this handle has launched (diagnostics; counts every launch). */
uint64_t trl_cuda_launch_count(trl_cuda_handle handle);

/* ---- failure injection (tests of the error paths; no counterpart in the reference) -------
 * trl_cuda_inject_alloc_failures: the handle's next `count` calls of trl_cuda_malloc fail with
 * TRL_ENOMEM (the device is not touched); 0 clears. trl_cuda_test_bounded_wait: enqueues a
 * kernel whose wait on a shared-memory barrier can never complete; the wait gives up after
 * `polls` polls (at most 2^24), the kernel returns, and the next
 * trl_cuda_synchronize reports TRL_ETIMEOUT, as every bounded device wait of this library
 * does. The handle stays usable. */
int trl_cuda_inject_alloc_failures(trl_cuda_handle handle, int count);
int trl_cuda_test_bounded_wait(trl_cuda_handle handle, unsigned polls);

/* FP64 tensor-core (DMMA m8n8k4) throughput of this GPU, measured with a loop of independent
 * DMMA chains on every SM (CUDA events; synchronises): the denominator of the contraction
 * kernels' tensor-pipe fraction. Diagnostics; no counterpart in the reference. */
int trl_cuda_measure_dmma_rate(trl_cuda_handle handle, double* host_tflops);

/* ---- per-kernel-class device timing ---------------------------------------------------
 * When enabled, every outermost C-ABI call is bracketed by CUDA events on the handle's
 * stream and credited with its algorithmic bytes (data each operand must move once) and
 * flops. Classes: spmm, block_dot, block_update, block_rotate, bv_mult, cholqr, bv_sub,
 * small_eigen, copy, sddmm, block_ops, reorth_pass2 (the conditional second Gram-Schmidt
 * pass of trl_cuda_project_out: time only, no bytes). */
#define TRL_PROF_CLASSES 12
typedef struct trl_kernel_stats {
  char name[24];
  uint64_t calls;
  double seconds;
  double bytes;
  double flops;
} trl_kernel_stats;
/* on != 0 starts collecting (and clears the totals); on == 0 stops. */
int trl_cuda_profile_enable(trl_cuda_handle handle, int on);
/* Synchronises the stream and copies the TRL_PROF_CLASSES totals into out. */
int trl_cuda_profile_read(trl_cuda_handle handle, trl_kernel_stats* out);

/* ---- memory (replaces aligned host allocation: multivector.hh:44-48, blockmatrix.hh:28-32)
 * Device memory from the handle's memory pool (256-byte aligned, usable from any stream on
 * return). The pool keeps freed memory reserved until the handle is destroyed, so repeated
 * solves reuse it instead of returning it to the driver. trl_cuda_free takes a block from
 * trl_cuda_malloc of the same handle and returns it to the pool in the order of the handle's
 * stream: work queued there before the call may still use it; work on other streams that
 * uses it must have finished. */
int trl_cuda_malloc(trl_cuda_handle handle, void** ptr, size_t bytes);
int trl_cuda_free(trl_cuda_handle handle, void* ptr);
/* Asynchronous copy on the handle's stream; TRL_D2H waits for completion before returning. */
int trl_cuda_memcpy(trl_cuda_handle handle, void* dst, const void* src, size_t bytes, int kind);
int trl_cuda_memset_zero(trl_cuda_handle handle, void* ptr, size_t bytes);

/* ---- block-vector kernels (trl::openmp::BlockView, impl/openmp/blockview.hh) ------- */

/* X = 0                                                        blockview.hh:31-36 */
int trl_cuda_bv_zero(trl_cuda_handle h, int dtype, void* X, int64_t n, int bs);
/* X = Y                                                        blockview.hh:59-63 */
int trl_cuda_bv_copy(trl_cuda_handle h, int dtype, void* X, const void* Y, int64_t n, int bs);
/* X -= Y                                                       blockview.hh:69-74 */
int trl_cuda_bv_sub(trl_cuda_handle h, int dtype, void* X, const void* Y, int64_t n, int bs);

enum trl_mult_mode {
  TRL_MULT = 0,           /* Y  = X W      blockview.hh:104-119 */
  TRL_MULT_TRANSPOSE = 1, /* Y  = X W^T    blockview.hh:126-141 */
  TRL_MULT_ADD = 2,       /* Y += X W      blockview.hh:81-97   */
  TRL_SUBTRACT = 3,       /* Y -= X W      blockview.hh:189-201 */
  TRL_SUBTRACT_TRANSPOSE = 4 /* Y -= X W^T  (a mult_transpose and a -= in one pass, lanczos.hh:243-245) */
};
/* Y (op)= X * W with W a device bs x bs FP64 block. The reference's
 * Xv.subtract_product(Yv, R) (Xv -= Yv R) is trl_cuda_bv_mult(h, dt, TRL_SUBTRACT, Yv, R, Xv, n, bs). */
int trl_cuda_bv_mult(trl_cuda_handle h, int dtype, int mode, const void* X, const double* W, void* Y, int64_t n, int bs);

/* Element-type conversion of `count` elements (FP64 <-> FP32; equal types copy). Used to
 * move Ritz vectors between the FP32 and FP64 phases of the mixed-precision solve. */
int trl_cuda_convert(trl_cuda_handle h, int dst_dtype, void* dst, int src_dtype, const void* src, int64_t count);

/* out (n x ncols row-major FP64) = the first ncols columns of the block-major multivector
 * X (nblk = ceil(ncols/bs) blocks of n x bs, FP64). */
int trl_cuda_unblock(trl_cuda_handle h, const double* X, int64_t n, int bs, int ncols, double* out);

/* Multi-block inner product: C_j = V_j^T W for j < nblk, V_j = V + j*n*bs.
 * C is nblk consecutive bs x bs FP64 blocks. nblk = 1 is BlockView::dot
 * (blockview.hh:152-182) and EVPBase::dot (evp_base.hh:37). Deterministic two-stage
 * reduction (the result does not depend on scheduling). */
int trl_cuda_block_dot(trl_cuda_handle h, int dtype, const void* V, int nblk, const void* W, int64_t n, int bs, double* C);

/* Allocation-free variant of trl_cuda_block_dot. It has no counterpart in the reference.
 *
 * For callers that may not allocate device memory: programs that hand all GPU memory to
 * their own pool allocator and do not let libraries call cudaMalloc behind their back, and
 * latency-critical loops that cannot afford an allocation or the device-wide
 * synchronisation that freeing one brings. It needs no handle either (creating a handle
 * allocates): pass the cudaStream_t to enqueue on and make the stream's device current.
 *
 * Computes the same C_j = V_j^T W (j < nblk) as trl_cuda_block_dot. Its partial sums go to
 * a fixed array inside this library (2 MiB of device memory on every GPU that loads the
 * library, held until the process exits), so nblk*bs*bs may be at most
 * TRL_CUDA_NOALLOC_MAX_ENTRIES; larger requests return TRL_EINVAL and do nothing.
 * The first call on each device looks up that array's device address (once per device, with
 * the device current); make that first call before any stream capture. All calls share the
 * one array: calls that may run at the same time on the GPU (different streams, or several
 * threads) race on it and must be serialised by the caller. The array's contents left by a
 * previous call are never read. The looked-up address is kept for the life of the process:
 * after cudaDeviceReset on a device this entry point is no longer valid on that device.
 * Returns TRL_OK, TRL_EINVAL, TRL_ENOTSUP or TRL_ECUDA (no error message is recorded). */
#define TRL_CUDA_NOALLOC_MAX_ENTRIES 16384
int trl_cuda_block_dot_noalloc(void* stream, int dtype, const void* V, int nblk, const void* W, int64_t n, int bs, double* C);

/* Projection update W -= sum_{j<nblk} V_j C_j (C as returned by trl_cuda_block_dot).
 * With trl_cuda_block_dot this is one classical Gram-Schmidt pass against nblk blocks,
 * replacing nblk rounds of ModifiedGS (reorthogonalization.hh:14-21). */
int trl_cuda_block_update(trl_cuda_handle h, int dtype, void* W, const void* V, int nblk, const double* C, int64_t n, int bs);

/* Classical Gram-Schmidt of W against V_0..V_{nblk-1}, fused for the reorthogonalisation
 * step of the driver (replaces ModifiedGS, reorthogonalization.hh:14-21):
 *   pass 1: C = V^T W (one multi-block dot), W -= V C (one update that also forms W^T W);
 *   pass 2 (W -= V (V^T W) again): always for TRL_CGS_TWO; for TRL_CGS_IFNEEDED only when
 *   a column kept less than `eta` of its norm through pass 1 (the DGKS criterion of
 *   Daniel, Gragg, Kaufman & Stewart, 1976; eta = 1/sqrt(2) is customary), decided on the
 *   device without a host round trip; never for TRL_CGS_ONE.
 * G (device, bs x bs) receives W^T W of the result, for trl_cuda_cholqr_gram. When W is the
 * block right after V_{nblk-1} (as in the driver) the Gram of the input rides along with
 * pass 1's dot. */
enum trl_cgs_mode { TRL_CGS_ONE = 0, TRL_CGS_TWO = 1, TRL_CGS_IFNEEDED = 2 };
int trl_cuda_project_out(trl_cuda_handle h, int dtype, const void* V, int nblk, void* W, int64_t n, int bs, int mode, double eta, double* G);

/* Partial reorthogonalisation (a ReorthogonalizationStrategy beyond the reference's full
 * ModifiedGS, reorthogonalization.hh:12-22): W is projected against the nblk blocks of V
 * only when a sketch says it has lost orthogonality to them. S (n x bs, same dtype) is a
 * random combination of those blocks, S = sum_j V_j G_j with G_j entries N(0, 1/bs), so
 * that ||S^T W||_F estimates ||V^T W||_F; when ||S^T W||_F > thr ||W||_F pass 1 of
 * TRL_CGS_IFNEEDED runs (and its DGKS second pass where needed), otherwise W is left as it
 * is. Decided on the device. G: the Gram matrix of the resulting W.
 * pair_state (device int, zero-initialised, kept by the caller across the steps of one
 * recurrence; NULL: off): a step whose sketch test fired also projects the next step. In a
 * three-term recurrence W_{i+1} inherits the loss of V_{i-1} through its B term, so
 * projecting one step alone leaves the loss to return two steps later (Simon's partial
 * reorthogonalisation projects pairs for the same reason). */
int trl_cuda_project_out_sketch(trl_cuda_handle h, int dtype, const void* V, int nblk, void* W, int64_t n, int bs, const void* S, double thr, double eta, double* G,
                                int* pair_state);

/* trl_cuda_cholqr with the Gram matrix of the first pass supplied (G0 = X^T X on the device,
 * e.g. from trl_cuda_project_out); each further pass forms its Gram matrix while it applies
 * U^{-1}, so CholQR2 reads and writes X twice. G0 == NULL is trl_cuda_cholqr. */
int trl_cuda_cholqr_gram(trl_cuda_handle h, int dtype, void* X, int64_t n, int bs, int passes, double* R, const double* G0);

/* Thick-restart rotation W_j = sum_{i<m} V_i Y(i,j) for j < k, in one pass over V.
 * Y is a block matrix with ldy block columns (Y(i,j) at Y + (i*ldy + j)*bs*bs).
 * Replaces the k*m BlockView::mult_add calls of lanczos.hh:105-114. W must not overlap V. */
int trl_cuda_block_rotate(trl_cuda_handle h, int dtype, const void* V, int m, const double* Y, int ldy, int k, void* W, int64_t n, int bs);

/* Cholesky-QR orthonormalisation in place: X <- X U^{-1} with X^T X = U^T U, repeated
 * `passes` times (1 = the reference's CholQR, evp_base.hh:39-71; 2 = CholQR2). On exit R
 * (device bs x bs FP64, upper triangular) satisfies X_in = X_out R. A non-positive pivot
 * leaves X and R unchanged for that pass and records TRL_ECHOLESKY. */
int trl_cuda_cholqr(trl_cuda_handle h, int dtype, void* X, int64_t n, int bs, int passes, double* R);

/* ---- sparse operator ------------------------------------------------------------- */

/* Y = alpha * A X + beta * X (X, Y: n x bs, dtype; A values may be FP64 or FP32).
 * alpha = 1, beta = 0 is CSREVP::apply (examples/sycl/csrevp.hh:159-187,
 * examples/openmp/csrevp.hh:36-44). X and Y must not overlap. */
int trl_cuda_spmm(trl_cuda_handle h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, double alpha, double beta);

/* Y = alpha * A X + beta * X + gamma * W (W: n x bs of dtype, may be Y itself, not X): the
 * three-term step of a Chebyshev filter in one pass. gamma = 0, W = NULL is trl_cuda_spmm.
 * No counterpart in the reference (used by the mixed-precision refinement). */
int trl_cuda_spmm3(trl_cuda_handle h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, double alpha, double beta, double gamma, const void* W);

/* trl_cuda_spmm3 on nb blocks at once: X, Y and W (or W = NULL) each hold nb consecutive
 * n x bs blocks; block j gets Y_j = alpha A X_j + beta X_j + gamma W_j. Each row group's CSR
 * entries are read once for all nb blocks. */
int trl_cuda_spmm_blocks(trl_cuda_handle h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, int nb, double alpha, double beta, double gamma, const void* W);

/* ---- prepared operator (the solver's SpMM) --------------------------------------------
 * The operator of CSREVP::apply (examples/sycl/csrevp.hh:159-187,
 * examples/openmp/csrevp.hh:36-44), converted once for repeated SpMMs with one block size:
 * a sliced-ELL copy (SELL-C-sigma) in which rows are sorted by length inside windows of 4096
 * rows and each slice of C rows (C = the rows one warp covers for the dtype and block size)
 * stores slot j of its C rows as C consecutive indices and values. Each row still sums its
 * entries in CSR order, as the per-row walk of trl_cuda_spmm_blocks does (bit-identical).
 * trl_cuda_op_create reads A (device CSR; its arrays are not referenced afterwards) and
 * allocates the copy from the handle's memory pool; it synchronises the stream once (to size
 * the copy). The op belongs to the handle's device and is released with
 * trl_cuda_op_destroy on the same handle. */
typedef struct trl_cuda_sell_op* trl_cuda_op;
int trl_cuda_op_create(trl_cuda_handle h, const trl_csr* A, int bs, trl_cuda_op* op);
int trl_cuda_op_destroy(trl_cuda_handle h, trl_cuda_op op);
/* Entries stored (padding included), slice height C and longest row (any may be NULL). */
int trl_cuda_op_info(trl_cuda_op op, int64_t* stored_entries, int* slice_height, int* longest_row);
/* Y_j = alpha A X_j + beta X_j + gamma W_j for j < nb (nb consecutive n x bs blocks of the
 * op's dtype; W may be NULL or Y itself, never X). nb = 1, gamma = 0, W = NULL is
 * CSREVP::apply with the shift beta; the multi-block form is one degree of a Chebyshev
 * filter on nb blocks. */
int trl_cuda_op_spmm(trl_cuda_handle h, trl_cuda_op op, const void* X, void* Y, int nb, double alpha, double beta, double gamma, const void* W);

/* Gershgorin interval of alpha*A + beta*I: *host_lo = min_i (c_i - r_i), *host_hi =
 * max_i (c_i + r_i), c_i = alpha*a_ii + beta, r_i = |alpha| sum_{j != i} |a_ij|. Contains
 * every eigenvalue. Synchronises the stream. */
int trl_cuda_csr_gershgorin(trl_cuda_handle h, const trl_csr* A, double alpha, double beta, double* host_lo, double* host_hi);

/* *host_out = max_i sum_j |alpha*a_ij + beta*delta_ij| (= ||alpha*A + beta*I||_1 for a
 * symmetric A; an upper bound of its 2-norm). Synchronises the stream. */
int trl_cuda_csr_norm1(trl_cuda_handle h, const trl_csr* A, double alpha, double beta, double* host_out);

/* Sampled dense-dense product over the CSR pattern (adjoint of the eigenvalues):
 * out[p] = sum_{c<k} w[c] * X[row(p), c] * X[col(p), c] for every stored entry p.
 * X: n x k row-major FP64 (device), w: k FP64 (device), out: nnz FP64 (device).
 * No counterpart in the reference (it has no derivatives). */
int trl_cuda_sddmm(trl_cuda_handle h, const trl_csr* pattern, const double* X, int k, const double* w, double* out);

/* Adjoint of a weighted eigenvalue sum f = sum_c w[c] lambda[c] with respect to the stored
 * entries of the operator (no counterpart in the reference, which has no derivatives).
 * X: n x k row-major FP64 (device), the eigenvectors, normalised in the problem's inner
 * product (x^T x = 1, or x^T M x = 1 for K x = lambda M x); host_evals / host_weights: k
 * values on the host. Eigenvalues closer than cluster_rtol * max|lambda| are one cluster;
 * inside a cluster the weights are replaced by their mean, which makes f's gradient
 * independent of the basis chosen inside the degenerate eigenspace (the projector of a
 * cluster is well defined; its individual eigenvectors are not).
 *   kind = 0: grad[p] = df/dA_ij  = sum_c wbar[c] x_c[i] x_c[j]            (A, or K)
 *   kind = 1: grad[p] = df/dM_ij  = -sum_c wbar[c] lambda[c] x_c[i] x_c[j] (mass M)
 * for every stored entry p = (i, j) of `pattern` (values unused). */
int trl_cuda_eigen_adjoint(trl_cuda_handle h, const trl_csr* pattern, const double* X, int k, const double* host_evals, const double* host_weights, double cluster_rtol,
                           int kind, double* grad);

/* ---- small bs x bs block operations (impl/openmp/matrixblockview.hh:30-74) ---------- */
int trl_cuda_mb_copy(trl_cuda_handle h, double* dst, const double* src, int bs, int transpose); /* :30-46 */
int trl_cuda_mb_zero(trl_cuda_handle h, double* dst, int bs);                                   /* :48-52 */
int trl_cuda_mb_mult(trl_cuda_handle h, const double* A, const double* B, double* C, int bs);   /* :54-67 C = A B */
/* dst(i,i) = host_values[i]; off-diagonal entries unchanged.                                    :69-74 */
int trl_cuda_mb_set_diagonal(trl_cuda_handle h, double* dst, const double* host_values, int bs);

/* ---- projected eigenproblem (EVPBase::solve_small_dense, evp_base.hh:79-154) ------ */
/* T: nblk x nblk block matrix (device; only its lower triangle is read). On return:
 * evals (device, N = nblk*bs) sorted by decreasing |theta|; evecs (device) the matching
 * eigenvectors in block-matrix layout (column c of the N x N matrix is eigenvector c);
 * host_evals (N doubles) a host copy of evals; *host_nconv the number of the first
 * min(nev, N) pairs whose Ritz estimate ||beta y_last|| / max(|theta|, eps) < tol.
 * Synchronises the stream. */
/* trl_cuda_small_eigen with eigenvectors for the first kvec pairs only (0 <= kvec <= N):
 * columns kvec.. of evecs are zero; evals, host_evals and *host_nconv (over the first
 * min(nev, kvec) pairs) as above. The driver reads only the kept kr = nev/bs + 1 blocks of
 * eigenvectors (lanczos.hh:105-131), so EVPBase::solve_small_dense asks for kr*bs. For
 * 3 <= N <= 448 and kvec <= 128 it runs on hand-written kernels: Householder
 * tridiagonalisation in one thread-block cluster, bisection, inverse iteration, and the
 * back-transform; otherwise it uses trl_cuda_small_eigen. Synchronises the stream. */
int trl_cuda_small_eigen_partial(trl_cuda_handle h, const double* T, int nblk, int bs, const double* beta, int nev, double tol, int kvec, double* evals,
                                 double* evecs, double* host_evals, int* host_nconv);
int trl_cuda_small_eigen(trl_cuda_handle h, const double* T, int nblk, int bs, const double* beta, int nev, double tol, double* evals, double* evecs,
                         double* host_evals, int* host_nconv);

#ifdef __cplusplus
}
#endif

#endif /* TRL_CUDA_H */
