// Small bs x bs block operations and the projected eigenproblem of the restart.
//
// The projected matrix T (N = nblk*bs <= a few thousand) stays on the device: it is
// assembled dense from its lower triangle (the reference's Eigen solver reads the lower
// triangle only, evp_base.hh:95), diagonalised by cuSOLVER's symmetric divide-and-conquer
// (syevd), re-ordered by decreasing |theta| (evp_base.hh:101-103) into the block layout,
// and the Ritz estimates ||beta * y_last|| / max(|theta|, eps) (evp_base.hh:124-151) are
// counted on the device. Only the eigenvalues and the converged count come back to the host.
#include "common.cuh"

#include <cusolverDn.h>

#include <cfloat>
#include <cstring>

namespace {

struct DiagValues {
  double v[16];
};

__global__ void k_mb_copy(double* __restrict__ dst, const double* __restrict__ src, int bs, int transpose)
{
  const int e = threadIdx.x;
  if (e >= bs * bs) return;
  const int i = e / bs, j = e % bs;
  dst[e] = transpose ? src[j * bs + i] : src[e];
}

__global__ void k_mb_mult(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C, int bs)
{
  const int e = threadIdx.x;
  if (e >= bs * bs) return;
  const int i = e / bs, j = e % bs;
  double s = 0.0;
  for (int k = 0; k < bs; ++k) s = fma(A[i * bs + k], B[k * bs + j], s);
  C[e] = s;
}

__global__ void k_mb_set_diag(double* __restrict__ dst, DiagValues d, int bs)
{
  const int i = threadIdx.x;
  if (i < bs) dst[i * bs + i] = d.v[i];
}

// dense column-major A (N x N) from the lower triangle of the block matrix T
__global__ void k_assemble_dense(const double* __restrict__ T, int nblk, int bs, double* __restrict__ A)
{
  const int N = nblk * bs;
  const int64_t total = static_cast<int64_t>(N) * N;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(e / N), r = static_cast<int>(e % N); // A[c*N + r] = M(r, c)
    const int hi = r > c ? r : c, lo = r > c ? c : r;
    const int bi = hi / bs, ri = hi % bs, bj = lo / bs, cj = lo % bs;
    A[e] = T[(static_cast<int64_t>(bi) * nblk + bj) * bs * bs + ri * bs + cj];
  }
}

// rank of each eigenvalue in decreasing |theta| order (ties keep ascending index)
__global__ void k_rank(const double* __restrict__ w, int N, int* __restrict__ perm, double* __restrict__ evals_sorted, const int* __restrict__ syevd_info, int* status)
{
  if (blockIdx.x == 0 && threadIdx.x == 0 && *syevd_info != 0) atomicOr(status, TRL_DEV_EIGEN);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double ai = fabs(w[i]);
    int r = 0;
    for (int j = 0; j < N; ++j) {
      const double aj = fabs(w[j]);
      r += (aj > ai) || (aj == ai && j < i);
    }
    perm[r] = i;
    evals_sorted[r] = w[i];
  }
}

__global__ void k_scatter_evecs(const double* __restrict__ A, const int* __restrict__ perm, int nblk, int bs, double* __restrict__ Y)
{
  const int N = nblk * bs;
  const int64_t total = static_cast<int64_t>(N) * N;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // Y in block layout: e = ((bi*nblk + bj)*bs + ri)*bs + cj
    const int cj = static_cast<int>(e % bs);
    const int64_t q = e / bs;
    const int ri = static_cast<int>(q % bs);
    const int64_t blk = q / bs;
    const int bj = static_cast<int>(blk % nblk), bi = static_cast<int>(blk / nblk);
    const int row = bi * bs + ri, col = bj * bs + cj;
    Y[e] = A[static_cast<int64_t>(perm[col]) * N + row];
  }
}

__global__ void k_count_converged(const double* __restrict__ A, const int* __restrict__ perm, const double* __restrict__ evals_sorted, const double* __restrict__ beta, int nblk,
                                  int bs, int ncheck, double tol, int* __restrict__ count)
{
  const int N = nblk * bs;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncheck; c += gridDim.x * blockDim.x) {
    const double* y = A + static_cast<int64_t>(perm[c]) * N + (nblk - 1) * bs;
    double nrm2 = 0.0;
    for (int i = 0; i < bs; ++i) {
      double s = 0.0;
      for (int k = 0; k < bs; ++k) s += beta[i * bs + k] * y[k];
      nrm2 += s * s;
    }
    const double denom = fmax(fabs(evals_sorted[c]), DBL_EPSILON);
    if (sqrt(nrm2) / denom < tol) atomicAdd(count, 1);
  }
}

} // namespace

using namespace trl_detail;

namespace trl_detail {

void* small_scratch(trl_cuda_context* h)
{
  if (!h->d_small) {
    if (cudaMalloc(&h->d_small, 1024 * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      h->d_small = nullptr;
      set_error(h, TRL_ENOMEM, "scratch allocation failed");
      return nullptr;
    }
  }
  return h->d_small;
}

void destroy_solver(trl_cuda_context* h)
{
  if (h->solver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(h->solver));
  if (h->syevd_work) cudaFree(h->syevd_work);
  h->solver = nullptr;
  h->syevd_work = nullptr;
  h->syevd_work_bytes = 0;
}

} // namespace trl_detail

extern "C" {

int trl_cuda_mb_copy(trl_cuda_handle h, double* dst, const double* src, int bs, int transpose)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || !dst || !src) return set_error(h, TRL_EINVAL, "bad block copy arguments");
  if (dst == src && !transpose) return TRL_OK;
  if (dst == src) return set_error(h, TRL_EINVAL, "in-place transpose not supported");
  ProfScope prof(h, PROF_BLOCK_OPS, 16.0 * bs * bs);
  k_mb_copy<<<1, bs * bs, 0, h->stream>>>(dst, src, bs, transpose);
  return after_launch(h, "mb_copy");
}

int trl_cuda_mb_zero(trl_cuda_handle h, double* dst, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || !dst) return set_error(h, TRL_EINVAL, "bad block zero arguments");
  ProfScope prof(h, PROF_BLOCK_OPS, 8.0 * bs * bs);
  return trl_cuda_memset_zero(h, dst, sizeof(double) * bs * bs);
}

int trl_cuda_mb_mult(trl_cuda_handle h, const double* A, const double* B, double* C, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || !A || !B || !C) return set_error(h, TRL_EINVAL, "bad block mult arguments");
  if (C == A || C == B) return set_error(h, TRL_EINVAL, "block mult output must not alias an input");
  ProfScope prof(h, PROF_BLOCK_OPS, 24.0 * bs * bs, 2.0 * bs * bs * bs);
  k_mb_mult<<<1, bs * bs, 0, h->stream>>>(A, B, C, bs);
  return after_launch(h, "mb_mult");
}

int trl_cuda_mb_set_diagonal(trl_cuda_handle h, double* dst, const double* host_values, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || !dst || !host_values) return set_error(h, TRL_EINVAL, "bad set_diagonal arguments");
  ProfScope prof(h, PROF_BLOCK_OPS, 8.0 * bs);
  DiagValues d{};
  for (int i = 0; i < bs; ++i) d.v[i] = host_values[i];
  k_mb_set_diag<<<1, 32, 0, h->stream>>>(dst, d, bs);
  return after_launch(h, "mb_set_diagonal");
}

int trl_cuda_small_eigen(trl_cuda_handle h, const double* T, int nblk, int bs, const double* beta, int nev, double tol, double* evals, double* evecs, double* host_evals,
                         int* host_nconv)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || nblk <= 0 || !T || !beta || !evals || !evecs || !host_evals || !host_nconv) return set_error(h, TRL_EINVAL, "bad small_eigen arguments");
  const int N = nblk * bs;
  if (N > 8192) return set_error(h, TRL_EINVAL, "projected problem too large (%d)", N);
  ProfScope prof(h, PROF_SMALL_EIGEN, 16.0 * N * N);
  cusolverStatus_t cs;
  if (!h->solver) {
    cusolverDnHandle_t sh;
    if (cusolverDnCreate(&sh) != CUSOLVER_STATUS_SUCCESS) return set_error(h, TRL_ECUDA, "cusolverDnCreate failed");
    h->solver = sh;
  }
  auto sh = static_cast<cusolverDnHandle_t>(h->solver);
  cusolverDnSetStream(sh, h->stream);

  // workspace: A (N*N) | w (N) | evals scratch | perm (N ints) | info | count
  const size_t a_bytes = sizeof(double) * static_cast<size_t>(N) * N;
  const size_t w_bytes = sizeof(double) * N;
  const size_t off_w = a_bytes;
  const size_t off_perm = off_w + w_bytes;
  const size_t off_info = off_perm + sizeof(int) * N + 64;
  const size_t total = off_info + 64;
  char* ws = static_cast<char*>(workspace(h, total));
  if (!ws) return TRL_ENOMEM;
  double* A = reinterpret_cast<double*>(ws);
  double* w = reinterpret_cast<double*>(ws + off_w);
  int* perm = reinterpret_cast<int*>(ws + off_perm);
  int* info = reinterpret_cast<int*>(ws + off_info);
  int* count = info + 1;

  int lwork = 0;
  cs = cusolverDnDsyevd_bufferSize(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, N, A, N, w, &lwork);
  if (cs != CUSOLVER_STATUS_SUCCESS) return set_error(h, TRL_ECUDA, "syevd_bufferSize failed (%d)", static_cast<int>(cs));
  const size_t need = sizeof(double) * static_cast<size_t>(lwork);
  if (need > h->syevd_work_bytes) {
    cudaStreamSynchronize(h->stream);
    if (h->syevd_work) cudaFree(h->syevd_work);
    h->syevd_work = nullptr;
    h->syevd_work_bytes = 0;
    if (cudaMalloc(&h->syevd_work, need) != cudaSuccess) {
      cudaGetLastError();
      return set_error(h, TRL_ENOMEM, "syevd workspace allocation failed");
    }
    h->syevd_work_bytes = need;
  }

  const unsigned g = grid_for(h, static_cast<int64_t>(N) * N, 256, 4);
  k_assemble_dense<<<g, 256, 0, h->stream>>>(T, nblk, bs, A);
  if (int st = after_launch(h, "assemble")) return st;
  cs = cusolverDnDsyevd(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, N, A, N, w, static_cast<double*>(h->syevd_work), lwork, info);
  if (cs != CUSOLVER_STATUS_SUCCESS) return set_error(h, TRL_ECUDA, "syevd failed (%d)", static_cast<int>(cs));
  k_rank<<<(N + 255) / 256, 256, 0, h->stream>>>(w, N, perm, evals, info, h->d_status);
  if (int st = after_launch(h, "rank")) return st;
  k_scatter_evecs<<<g, 256, 0, h->stream>>>(A, perm, nblk, bs, evecs);
  if (int st = after_launch(h, "scatter")) return st;
  cudaMemsetAsync(count, 0, sizeof(int), h->stream);
  const int ncheck = nev < N ? nev : N;
  if (ncheck > 0) {
    k_count_converged<<<(ncheck + 127) / 128, 128, 0, h->stream>>>(A, perm, evals, beta, nblk, bs, ncheck, tol, count);
    if (int st = after_launch(h, "count")) return st;
  }
  char* pin = static_cast<char*>(pinned(h, w_bytes + 64));
  if (!pin) return TRL_ENOMEM;
  cudaMemcpyAsync(pin, evals, w_bytes, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(pin + w_bytes, count, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  int st = trl_cuda_synchronize(h);
  if (st) return st;
  std::memcpy(host_evals, pin, w_bytes);
  std::memcpy(host_nconv, pin + w_bytes, sizeof(int));
  return TRL_OK;
}

} // extern "C"
