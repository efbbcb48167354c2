/* trl_solver.h — C entry points that run trl's unchanged BlockLanczos driver
 * (include/trl/eigensolvers/lanczos.hh in the reference) on the CUDA backend
 * (include/trl/impl/cuda/, C ABI in trl_cuda.h) for a CSR operator.
 *
 * These replace the reference's example driver (examples/openmp/csrtest.cc:90-109: build a
 * CSR eigenproblem, fill initial_block(), solve(), read get_current_eigenvalues()) for
 * callers that are not C++ (ctypes, FFI) and add what the driver leaves out: Ritz vectors,
 * true residuals, per-phase device timings, and the mixed-precision mode.
 *
 * Modes
 *   TRL_MODE_FP64   FP64 basis, FP64 SpMM (the plain backend).
 *   TRL_MODE_FP32   FP32 basis and FP32 SpMM; Grams, Cholesky, the projected eigenproblem
 *                   and residuals in FP64. Accuracy is limited by FP32 storage.
 *   TRL_MODE_MIXED  TRL_MODE_FP32 to fp32_tol, then an FP64 refinement of the FP32 phase's
 *                   kept Ritz vectors (nev/bs + 1 blocks, widened to FP64) to `tol`:
 *                   TRL_REFINE_CHEBYSHEV: Rayleigh-Ritz on those vectors
 *                     alternated with Chebyshev-filtered subspace iteration on them (the
 *                     filter damps the spectrum beyond the kept Ritz values: the interval
 *                     from the far Gershgorin bound to them when they lie on one side of
 *                     zero, [-b, b] with b their smallest magnitude when they straddle it);
 *                   TRL_REFINE_LANCZOS: a random combination of them starts an FP64
 *                     BlockLanczos solve.
 *
 * The operator is alpha*A + beta*I (alpha = 1, beta = 0 for A itself).
 * Eigenpairs are returned in the driver's order: decreasing |theta| (evp_base.hh:103).
 */
#ifndef TRL_SOLVER_H
#define TRL_SOLVER_H

#include "trl_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

enum trl_mode { TRL_MODE_FP64 = 0, TRL_MODE_FP32 = 1, TRL_MODE_MIXED = 2 };
/* Reorthogonalisation strategy: the reference's ModifiedGS, or the backend's block classical
 * Gram-Schmidt variants (include/trl/impl/cuda/reorthogonalization.hh). */
enum trl_reorth { TRL_REORTH_MGS = 0, TRL_REORTH_CGS2 = 1, TRL_REORTH_CGS_IFNEEDED = 2, TRL_REORTH_CGS1 = 3, TRL_REORTH_PARTIAL = 4 };
/* FP64 refinement of the mixed mode. TRL_REFINE_AUTO (default): the Chebyshev refinement
 * after its first Rayleigh-Ritz step predicts its own time (degrees to the tolerance at the
 * predicted rate x one measured multi-block SpMM and a share of one measured
 * re-orthonormalisation; a two-sided filter, for kept values on both sides of zero, with a
 * 4x margin) and hands over to the Lanczos refinement when that is predicted cheaper
 * (estimated from the FP32 phase's time and the orders of magnitude left). */
enum trl_refine { TRL_REFINE_LANCZOS = 0, TRL_REFINE_CHEBYSHEV = 1, TRL_REFINE_AUTO = 2 };

typedef struct trl_solve_params {
  int bs;                        /* block size: 1, 2, 4, 8, 16 */
  int mode;                      /* trl_mode */
  unsigned nev;                  /* wanted eigenpairs */
  unsigned ncv;                  /* basis size in vectors (a multiple of bs) */
  unsigned max_restarts;         /* EigensolverParams::max_restarts (params.hh:8) */
  double tol;                    /* EigensolverParams::tolerance (params.hh:9) */
  double alpha, beta;            /* operator alpha*A + beta*I */
  int reorth;                    /* trl_reorth: reference ModifiedGS or block CGS2 */
  int cholqr_passes;             /* 1 = CholQR (reference), 2 = CholQR2 */
  double fp32_tol;               /* TRL_MODE_MIXED: tolerance of the FP32 phase */
  unsigned refine_max_restarts;  /* TRL_MODE_MIXED: max_restarts of the FP64 phase */
  int want_vectors;              /* form Ritz vectors and true residuals */
  int batching;                  /* fuse the restart rotation (see trl::cuda::Context) */
  unsigned seed;                 /* seed of the refinement's random combination */
  int refine;                    /* trl_refine (TRL_MODE_MIXED) */
  unsigned fp32_ncv;             /* TRL_MODE_MIXED: basis size of the FP32 phase (0: ncv) */
  int refine_fp32;               /* TRL_REFINE_CHEBYSHEV: filter in FP32 while the residual is
                                    above ~2e-5, then in FP64 (0: FP64 only) */
  int small_eigen_full;          /* 1: every eigenvector of the projected problem (cuSOLVER
                                    syevd); 0: the kept blocks' only (trl_cuda_small_eigen_partial) */
  double partial_threshold;      /* TRL_REORTH_PARTIAL: orthogonality loss ||V^T w|| / ||w||
                                    (sketch estimate) that triggers a projection (0: 1e-12;
                                    FP32 phases 1e-6 at least) */
  int partial_pairs;             /* TRL_REORTH_PARTIAL: a step whose sketch test fired also
                                    projects the next step (1, default; 0: that step only) */
} trl_solve_params;

typedef struct trl_solve_info {
  int converged;
  unsigned restarts;        /* restarts of the final phase */
  unsigned n_op_apply;      /* operator applications of the final phase */
  unsigned restarts_fp32;   /* TRL_MODE_MIXED: restarts of the FP32 phase */
  unsigned n_op_apply_fp32; /* TRL_MODE_MIXED: applications of the FP32 phase */
  double seconds;           /* device time (CUDA events) of the whole solve */
  double seconds_fp32;      /* device time of the FP32 phase (mixed) */
  double seconds_vectors;   /* device time of Ritz vectors + residuals */
  double max_rel_residual;  /* max_c ||op x_c - theta_c x_c|| / ||op||_1 (want_vectors) */
  double max_theta_residual;/* max_c ||op x_c - theta_c x_c|| / |theta_c| (want_vectors) */
  double op_norm1;          /* ||op||_1 = max row sum of |alpha*A + beta*I| */
  unsigned long long kernel_launches; /* kernels launched by the backend during the call */
  double h2d_bytes, d2h_bytes;        /* host<->device traffic of the call */
  unsigned refine_rounds;   /* Chebyshev refinement: Rayleigh-Ritz rounds (0: not run; 1 with
                               refine_used = TRL_REFINE_LANCZOS: handed over after its first) */
  unsigned refine_degree;   /* Chebyshev refinement: total filter degree */
  unsigned refine_degree_fp32; /* Chebyshev refinement: of which applied in FP32 */
  int refine_used;              /* TRL_MODE_MIXED: the refinement that ran (trl_refine) */
  double refine_predicted_s;    /* TRL_REFINE_AUTO: the Chebyshev refinement's predicted time */
  double refine_lanczos_estimate_s; /* TRL_REFINE_AUTO: the Lanczos refinement's estimated time */
} trl_solve_info;

void trl_solve_params_default(trl_solve_params* p);

/* Host in, host out: uploads the CSR operator and X0 (n x bs row-major), solves, and
 * returns evals[nev], optionally evecs (n x nev row-major) and resid[nev]
 * (||op x - theta x|| / ||op||_1). Runs on a handle of its own on `device`, created by the
 * first call and kept until the process exits together with the device memory its pool
 * holds (the peak of the calls so far), so that later calls reuse it; calls on one device
 * are serialised. */
int trl_solve_csr_host(const trl_solve_params* p, int device, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind, const double* values, const double* X0,
                       double* evals, double* evecs, double* resid, trl_solve_info* info);

/* Device-resident: A64 (FP64 values) is always needed; A32 (FP32 values of the same
 * pattern) is used by the FP32 / mixed modes and may be NULL for TRL_MODE_FP64.
 * X0 is n x bs FP64 on the device. evals_host[nev]; evecs_dev (n x nev row-major FP64,
 * device) and resid_host[nev] may be NULL. Synchronises the handle's stream on return. */
int trl_solve_csr_device(trl_cuda_handle h, const trl_solve_params* p, const trl_csr* A64, const trl_csr* A32, const double* X0, double* evals_host, double* evecs_dev,
                         double* resid_host, trl_solve_info* info);

/* Eigenpairs of an operator that is self-adjoint in the inner product <x, y> = x^T M y (M SPD,
 * device CSR, FP64), e.g. op = M^{-1} K for K x = lambda M x: BlockLanczos with dot(V, W) =
 * V^T (M W) and Cholesky-QR in that inner product, as the reference's generalised example
 * (examples/openmp/csrevp.hh:52-109, whose operator is (A - sigma B)^{-1} B through a sparse
 * LU; here the operator is given as a CSR matrix). FP64 only (p->mode = TRL_MODE_FP64);
 * eigenvectors are M-orthonormal; resid = ||op x - theta x||_2 / (||op||_1 ||x||_2). */
int trl_solve_csr_minner_device(trl_cuda_handle h, const trl_solve_params* p, const trl_csr* op, const trl_csr* M, const double* X0, double* evals_host, double* evecs_dev,
                                double* resid_host, trl_solve_info* info);

const char* trl_solver_last_error(void);

/* Matrix Market coordinate file -> CSR in full storage, in host memory allocated with
 * malloc (free with trl_csr_free_host). Replaces the reference's loader
 * (examples/sycl/csrevp.hh:26-124) with its semantics: a "symmetric" header mirrors every
 * off-diagonal entry (the mirror right after it), indices are 1-based in the file, entries
 * of a row keep their order in the file, duplicates are kept. Also reads "integer" and
 * "pattern" (value 1) files. `threads` host threads parse the data (<= 0: all cores).
 * TRL_EINVAL on a malformed file (message in trl_solver_last_error). */
int trl_csr_read_mtx(const char* path, int threads, int64_t* n_rows, int64_t* n_cols, int64_t* nnz, int32_t** rowptr, int32_t** colind, double** values);
void trl_csr_free_host(int32_t* rowptr, int32_t* colind, double* values);

#ifdef __cplusplus
}
#endif

#endif /* TRL_SOLVER_H */
