// Small bs x bs block operations and the projected eigenproblem of the restart.
//
// The projected matrix T (N = nblk*bs <= a few thousand) stays on the device: it is
// assembled dense from its lower triangle (the reference's Eigen solver reads the lower
// triangle only, evp_base.hh:95), diagonalised by cuSOLVER's symmetric divide-and-conquer
// (syevd), re-ordered by decreasing |theta| (evp_base.hh:101-103) into the block layout,
// and the Ritz estimates ||beta * y_last|| / max(|theta|, eps) (evp_base.hh:124-151) are
// counted on the device. Only the eigenvalues and the converged count come back to the host.
#include "common.cuh"

#include <cooperative_groups.h>
#include <cusolverDn.h>

#include <cfloat>
#include <cstring>
#include <mutex>

namespace {

struct DiagValues {
  double v[16];
};

__global__ void k_mb_copy(double* __restrict__ dst, const double* __restrict__ src, int bs, int transpose)
{
  ::trl_detail::pdl_enter();
  const int e = threadIdx.x;
  if (e >= bs * bs) return;
  const int i = e / bs, j = e % bs;
  dst[e] = transpose ? src[j * bs + i] : src[e];
}

__global__ void k_mb_mult(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C, int bs)
{
  ::trl_detail::pdl_enter();
  const int e = threadIdx.x;
  if (e >= bs * bs) return;
  const int i = e / bs, j = e % bs;
  double s = 0.0;
  for (int k = 0; k < bs; ++k) s = fma(A[i * bs + k], B[k * bs + j], s);
  C[e] = s;
}

__global__ void k_mb_set_diag(double* __restrict__ dst, DiagValues d, int bs)
{
  ::trl_detail::pdl_enter();
  const int i = threadIdx.x;
  if (i < bs) dst[i * bs + i] = d.v[i];
}

// max |T_ij| over the block matrix (one CTA) into *out
__global__ void __launch_bounds__(1024) k_max_abs(const double* __restrict__ T, int64_t count, double* __restrict__ out)
{
  ::trl_detail::pdl_enter();
  __shared__ double red[32];
  double m = 0.0;
  for (int64_t e = threadIdx.x; e < count; e += blockDim.x) m = fmax(m, fabs(T[e]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) *out = m;
  }
}

// Entries below kFlushRel * max|T| are set to zero when the dense copy is assembled: they
// change no eigenvalue by more than N * 1e-30 * ||T||, far below rounding, while leaving
// them in lets their squares underflow inside the Householder reduction (a converged Ritz
// pair's coupling in a thick-restart matrix can be ~1e-160 next to entries of order 10);
// a reflector built from an underflowed norm is not orthogonal, and the computed spectrum is
// then wrong (cuSOLVER's syevd on the GPU fails the same way on such matrices).
constexpr double kFlushRel = 1e-30;

// dense column-major A (N x N) from the lower triangle of the block matrix T
__global__ void k_assemble_dense(const double* __restrict__ T, int nblk, int bs, const double* __restrict__ tmax, double* __restrict__ A)
{
  ::trl_detail::pdl_enter();
  const int N = nblk * bs;
  const int64_t total = static_cast<int64_t>(N) * N;
  const double floor = kFlushRel * *tmax;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(e / N), r = static_cast<int>(e % N); // A[c*N + r] = M(r, c)
    const int hi = r > c ? r : c, lo = r > c ? c : r;
    const int bi = hi / bs, ri = hi % bs, bj = lo / bs, cj = lo % bs;
    const double v = T[(static_cast<int64_t>(bi) * nblk + bj) * bs * bs + ri * bs + cj];
    A[e] = fabs(v) < floor ? 0.0 : v;
  }
}

// rank of each eigenvalue in decreasing |theta| order (ties keep ascending index)
__global__ void k_rank(const double* __restrict__ w, int N, int* __restrict__ perm, double* __restrict__ evals_sorted, const int* __restrict__ syevd_info, int* status)
{
  ::trl_detail::pdl_enter();
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
  ::trl_detail::pdl_enter();
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
  ::trl_detail::pdl_enter();
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
    // zeroed once: the CholQR factor's ticket counter (doubles 768..) must start at zero
    cudaMemsetAsync(h->d_small, 0, 1024 * sizeof(double), h->stream);
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
  launch(k_mb_copy, 1, bs * bs, 0, h->stream, dst, src, bs, transpose);
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
  launch(k_mb_mult, 1, bs * bs, 0, h->stream, A, B, C, bs);
  return after_launch(h, "mb_mult");
}

int trl_cuda_mb_set_diagonal(trl_cuda_handle h, double* dst, const double* host_values, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || !dst || !host_values) return set_error(h, TRL_EINVAL, "bad set_diagonal arguments");
  ProfScope prof(h, PROF_BLOCK_OPS, 8.0 * bs);
  DiagValues d{};
  for (int i = 0; i < bs; ++i) d.v[i] = host_values[i];
  launch(k_mb_set_diag, 1, 32, 0, h->stream, dst, d, bs);
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
  const size_t off_tmax = (off_info + 64 + 15) / 16 * 16; // a double: 8-byte aligned whatever N is
  const size_t total = off_tmax + 64;
  char* ws = static_cast<char*>(workspace(h, total));
  if (!ws) return TRL_ENOMEM;
  double* A = reinterpret_cast<double*>(ws);
  double* w = reinterpret_cast<double*>(ws + off_w);
  int* perm = reinterpret_cast<int*>(ws + off_perm);
  int* info = reinterpret_cast<int*>(ws + off_info);
  int* count = info + 1;
  double* tmax = reinterpret_cast<double*>(ws + off_tmax);

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
  launch(k_max_abs, 1, 1024, 0, h->stream, T, static_cast<int64_t>(N) * N, tmax);
  launch(k_assemble_dense, g, 256, 0, h->stream, T, nblk, bs, tmax, A);
  if (int st = after_launch(h, "assemble")) return st;
  cs = cusolverDnDsyevd(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, N, A, N, w, static_cast<double*>(h->syevd_work), lwork, info);
  if (cs != CUSOLVER_STATUS_SUCCESS) return set_error(h, TRL_ECUDA, "syevd failed (%d)", static_cast<int>(cs));
  launch(k_rank, (N + 255) / 256, 256, 0, h->stream, w, N, perm, evals, info, h->d_status);
  if (int st = after_launch(h, "rank")) return st;
  launch(k_scatter_evecs, g, 256, 0, h->stream, A, perm, nblk, bs, evecs);
  if (int st = after_launch(h, "scatter")) return st;
  cudaMemsetAsync(count, 0, sizeof(int), h->stream);
  const int ncheck = nev < N ? nev : N;
  if (ncheck > 0) {
    launch(k_count_converged, (ncheck + 127) / 128, 128, 0, h->stream, A, perm, evals, beta, nblk, bs, ncheck, tol, count);
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

// ---- the projected eigenproblem for the eigenvectors the restart keeps ------------------
//
// trl_cuda_small_eigen_partial returns every eigenvalue but only the first kvec eigenvectors
// (|theta| descending), which is all the driver reads (the kept blocks, lanczos.hh:105-131).
// For 3 <= N <= kTriMaxN and kvec <= kTriMaxVec it runs without cuSOLVER:
//  1. k_tridiag: Householder tridiagonalisation Q^T A Q = T in ONE thread-block cluster of
//     8 or 16 CTAs. A (full symmetric storage) is distributed over the CTAs by rows (row g
//     on CTA g % C, in its shared memory up to N = 640); each step exchanges the Householder column and the
//     vector p = tau A v through distributed shared memory, two cluster barriers per step.
//     (cuSOLVER's tridiagonalisation of the same matrix is a sequence of small kernels, about
//     3.7 ms at N = 384 on B200.)
//  2. k_bisect: all eigenvalues of T by bisection on Sturm counts, one warp per eigenvalue,
//     each lane evaluating one of 32 points of the interval per iteration (multisection).
//  3. k_tri_factor / k_tri_solve / k_tri_gs: eigenvectors of T for the kvec selected
//     eigenvalues by inverse iteration (partial-pivoting LU of T - lambda I, tiny pivots
//     replaced by eps * ||T||), all vectors at once, then classical Gram-Schmidt applied
//     twice in ascending eigenvalue order. A solve shrinks the component along an eigenvalue
//     at distance g by eps * ||T|| / g relative to the wanted one, so three solves separate
//     every pair with g above ~1e-10 ||T|| to working accuracy; closer pairs (and exactly
//     equal ones) span their eigenspace and the Gram-Schmidt step makes them orthonormal.
//     The wanted end of a Lanczos T is one tight cluster (48 values within 5e-4 ||T|| at the
//     96^3 workload), so vectors are not iterated one after another.
//  4. k_wy_factor / k_backtransform: x = Q z with the stored reflectors in compact WY
//     chunks (Q restricted to a chunk = I - V T V^T).
// Otherwise it falls back to trl_cuda_small_eigen and zeroes the columns from kvec on.

namespace {

// The tridiagonalisation runs in one thread-block cluster; its rows live in the CTAs' shared
// memory while they fit, in global memory (the dense copy it works on, L2-resident) beyond:
//   N <= kTriMaxN8      8 CTAs (portable cluster size), rows in shared memory;
//   N <= kTriMaxN16    16 CTAs (non-portable cluster size), rows in shared memory;
//   N <= kTriMaxN      16 CTAs, rows in global memory.
// Rows per CTA * N * 8 B must fit one CTA's shared memory (227 KB) for the first two.
constexpr int kTriThreads = 512;
constexpr double kTinyNorm2 = 1e-290; // squared column norms below this are treated as zero
constexpr int kTriMaxN8 = 448;
constexpr int kTriMaxN16 = 640;
constexpr int kTriMaxN = 1024;
constexpr int kTriMaxVec = 256;    // vectors by inverse iteration
constexpr int kTriIters = 3;       // inverse-iteration sweeps
constexpr int kBisectMaxN = kTriMaxN;
constexpr size_t kTriGsMaxBytes = 200 * 1024; // the K vectors of N entries in one CTA's shared memory (else in global memory)

size_t tridiag_smem(int N, int C, bool global_rows)
{
  const int RB = (N + C - 1) / C;
  return sizeof(double) * ((global_rows ? 0 : static_cast<size_t>(RB) * N) + 4 * N + 2 * C * (kTriThreads / 32) + 8);
}

__device__ __forceinline__ double warp_sum(double v)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block sum over kTriThreads threads; `red` holds 32 doubles; all threads get the result
__device__ double block_sum(double v, double* red)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads(); // red may still be read from a previous call
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (warp == 0) {
    s = lane < static_cast<int>(blockDim.x >> 5) ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) red[0] = s;
  }
  __syncthreads();
  return red[0];
}

// dst[i] = src[i], i < count, by all threads of the CTA with kStageBatch global loads in
// flight per thread (a plain copy loop waits for each load before its store)
constexpr int kStageBatch = 8;

__device__ __forceinline__ void stage(double* dst, const double* __restrict__ src, int count)
{
  const int step = static_cast<int>(blockDim.x);
  for (int base = threadIdx.x; base < count; base += step * kStageBatch) {
    double v[kStageBatch];
#pragma unroll
    for (int u = 0; u < kStageBatch; ++u) {
      const int i = base + u * step;
      v[u] = i < count ? src[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kStageBatch; ++u) {
      const int i = base + u * step;
      if (i < count) dst[i] = v[u];
    }
  }
}

// A: N x N symmetric (full storage). Outputs: d[N], e[N-1] of T = Q^T A Q with
// Q = H_0 ... H_{N-3}, H_k = I - tau_k v_k v_k^T, v_k stored in refl[k*N + k+1 .. N-1]
// (refl[k*N + k+1] = 1). Row g belongs to CTA g % C of the cluster (C CTAs); with
// kGlobalRows it is updated in place in A (only its owner reads or writes it, so the CTA's
// own barriers order the accesses), otherwise it is copied into the owner's shared memory.
// Exchange by pushing: before each cluster barrier every CTA stores its entries of the
// Householder column (then of p = tau A v) and its per-warp partial sums into the shared
// memory of every CTA of the cluster (st.shared::cluster through map_shared_rank); after
// the barrier each CTA reads only its own shared memory. Every CTA reduces the same
// partials in the same order, so all hold bit-identical scalars. A buffer filled at one
// barrier is read before the next one, which its next writers wait for.
template <int C, bool kGlobalRows>
__global__ void __launch_bounds__(kTriThreads, 1)
    k_tridiag(double* __restrict__ A, int N, double* __restrict__ dout, double* __restrict__ eout, double* __restrict__ tau_out, double* __restrict__ refl)
{
  ::trl_detail::pdl_enter();
  namespace cg = cooperative_groups;
  constexpr int NW = kTriThreads / 32;
  constexpr int NP = C * NW; // partials per exchange
  static_assert(NP % 32 == 0, "partials are reduced as NP / 32 per lane");
  cg::cluster_group cluster = cg::this_cluster();
  const int r = static_cast<int>(cluster.block_rank());
  const int RB = (N + C - 1) / C;
  extern __shared__ __align__(16) double sm[];
  double* const rows = kGlobalRows ? nullptr : sm; // RB x N, local row l = global row r + C * l
  double* xfull = sm + (kGlobalRows ? 0 : RB * N); // N: column k below the diagonal (pushed by the owners)
  double* pfull = xfull + N;      // N: p (pushed by the owners)
  double* vfull = pfull + N;      // N
  double* wfull = vfull + N;      // N
  double* part = wfull + N;       // NP sums of squares (slot rank * NW + warp), then x0
  double* part2 = part + NP + 8;  // NP partial p.v
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto row = [&](int l) -> double* { return kGlobalRows ? A + static_cast<size_t>(r + C * l) * N : rows + static_cast<size_t>(l) * N; };

  auto local_sum = [&](const double* slot) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < NP / 32; ++q) s += slot[lane + 32 * q];
    return warp_sum(s);
  };
  // store v at offset `at` of `buf` in every CTA of the cluster
  auto push = [&](double* buf, int at, double v) {
#pragma unroll
    for (int q = 0; q < C; ++q) cluster.map_shared_rank(buf, q)[at] = v;
  };

  if (!kGlobalRows) {
    for (int l = 0; l < RB; ++l) {
      const int g = r + C * l;
      if (g < N) stage(rows + l * N, A + static_cast<size_t>(g) * N, N);
      else
        for (int j = tid; j < N; j += kTriThreads) rows[l * N + j] = 0.0;
    }
  }
  cluster.sync(); // every CTA is running before any pushes into it

  for (int k = 0; k < N - 2; ++k) {
    const int l0 = (k + 1 - r + C - 1) / C > 0 ? (k + 1 - r + C - 1) / C : 0; // first local row > k
    if (r == k % C && tid == 0) dout[k] = row(k / C)[k];
    // ---- phase A: push this CTA's entries of x = A[k+1:, k] and its partial sum of squares
    {
      double ssq = 0.0;
      if (tid < RB - l0) {
        const int l = l0 + tid, g = r + C * l;
        if (g < N) {
          const double x = row(l)[k];
          push(xfull, g, x);
          if (g > k + 1) ssq = x * x;
        }
      }
      ssq = warp_sum(ssq);
      if (lane < C) cluster.map_shared_rank(part, lane)[r * NW + warp] = ssq;
      if (tid == 0 && r == (k + 1) % C) push(part, NP, row((k + 1) / C)[k]);
    }
    cluster.sync(); // #1
    const double xnorm2 = local_sum(part);
    const double x0 = part[NP];
    double tau = 0.0, beta = x0, scale = 0.0;
    // a column whose squares underflow is left as it is (H = I): a reflector built from a
    // norm computed in the subnormal range would not be orthogonal
    if (xnorm2 > 0.0 && x0 * x0 + xnorm2 > kTinyNorm2) {
      beta = -copysign(sqrt(x0 * x0 + xnorm2), x0);
      tau = (beta - x0) / beta;
      scale = 1.0 / (x0 - beta);
    }
    for (int j = k + 1 + tid; j < N; j += kTriThreads) vfull[j] = (j == k + 1) ? 1.0 : xfull[j] * scale;
    __syncthreads();
    if (r == k % C) {
      for (int j = k + 1 + tid; j < N; j += kTriThreads) refl[static_cast<size_t>(k) * N + j] = vfull[j];
      if (tid == 0) {
        tau_out[k] = tau;
        eout[k] = beta;
      }
    }
    // ---- phase C: p = tau * A_trail v for this CTA's rows (warp per row), pushed with the
    // partial p.v
    double pv = 0.0;
    for (int l = l0 + warp; l < RB; l += NW) {
      const int g = r + C * l;
      if (g >= N) break;
      const double* rl = row(l);
      double s = 0.0;
      for (int j = k + 1 + lane; j < N; j += 32) s = fma(rl[j], vfull[j], s);
      s = warp_sum(s) * tau;
      if (lane < C) cluster.map_shared_rank(pfull, lane)[g] = s;
      pv = fma(s, vfull[g], pv);
    }
    if (lane < C) cluster.map_shared_rank(part2, lane)[r * NW + warp] = pv;
    cluster.sync(); // #2
    const double K = 0.5 * tau * local_sum(part2);
    for (int j = k + 1 + tid; j < N; j += kTriThreads) wfull[j] = pfull[j] - K * vfull[j];
    __syncthreads();
    // ---- phase D: rank-2 update of this CTA's trailing rows (warp per row)
    if (tau != 0.0) {
      for (int l = l0 + warp; l < RB; l += NW) {
        const int g = r + C * l;
        if (g >= N) break;
        double* rl = row(l);
        const double vg = vfull[g], wg = wfull[g];
        for (int j = k + 1 + lane; j < N; j += 32) rl[j] -= vg * wfull[j] + wg * vfull[j];
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (N >= 2 && r == (N - 2) % C) dout[N - 2] = row((N - 2) / C)[N - 2];
    if (r == (N - 1) % C) {
      dout[N - 1] = row((N - 1) / C)[N - 1];
      if (N >= 2) eout[N - 2] = row((N - 1) / C)[N - 2];
    }
  }
  cluster.sync(); // no CTA leaves while another may still store into its shared memory
}

// number of eigenvalues of the tridiagonal (d, e2 = e^2) below sigma
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int N, double sigma, double pivmin)
{
  double q = d[0] - sigma;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q < 0.0;
  for (int j = 1; j < N; ++j) {
    q = (d[j] - sigma) - e2[j - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < 0.0;
  }
  return c;
}

// w[i] = i-th smallest eigenvalue of the tridiagonal (d, e); one warp per eigenvalue
__global__ void __launch_bounds__(256) k_bisect(const double* __restrict__ dg, const double* __restrict__ eg, int N, double* __restrict__ w)
{
  ::trl_detail::pdl_enter();
  __shared__ double d[kBisectMaxN], e2[kBisectMaxN];
  __shared__ double bounds[3];
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    d[j] = dg[j];
    e2[j] = j + 1 < N ? eg[j] * eg[j] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double lo = d[0], hi = d[0], emax = 0.0;
    for (int j = 0; j < N; ++j) {
      const double rad = (j > 0 ? sqrt(e2[j - 1]) : 0.0) + (j + 1 < N ? sqrt(e2[j]) : 0.0);
      lo = fmin(lo, d[j] - rad);
      hi = fmax(hi, d[j] + rad);
      if (j + 1 < N) emax = fmax(emax, e2[j]);
    }
    const double nrm = fmax(fabs(lo), fabs(hi));
    bounds[0] = lo - 2.0 * DBL_EPSILON * nrm * N - DBL_MIN;
    bounds[1] = hi + 2.0 * DBL_EPSILON * nrm * N + DBL_MIN;
    bounds[2] = DBL_MIN * fmax(1.0, emax); // pivmin
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= N) return;
  double lo = bounds[0], hi = bounds[1];
  const double pivmin = bounds[2];
  for (int it = 0; it < 64; ++it) {
    const double width = hi - lo;
    if (width <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 2.0 * pivmin) break;
    const double sigma = lo + width * (lane + 1) / 33.0;
    const int c = sturm_count(d, e2, N, sigma, pivmin);
    // smallest lane whose point has more than i eigenvalues below it
    const unsigned above = __ballot_sync(0xffffffffu, c > i);
    const int q = above ? __ffs(above) - 1 : 32;
    const double nlo = q == 0 ? lo : lo + width * q / 33.0;
    const double nhi = q == 32 ? hi : lo + width * (q + 1) / 33.0;
    if (!(nhi < hi || nlo > lo)) break; // no progress in floating point
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) w[i] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double hash_unit(unsigned a, unsigned b)
{
  unsigned x = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
  x ^= x >> 15;
  x *= 0x2C1B3C6Du;
  x ^= x >> 12;
  x *= 0x297A2D39u;
  x ^= x >> 15;
  return (static_cast<double>(x) / 4294967295.0) * 2.0 - 1.0;
}

// Inverse iteration for the eigenvectors of the tridiagonal (d, e) at the K eigenvalues
// w[sel[t]] (sel ascending). Vectors: Z[t * N + i]. Per vector t the factorisation
// P L U = T - lambda_t I (general tridiagonal LU with partial pivoting; pivots below
// eps * ||T|| replaced by +-eps * ||T||) is stored as F[t][5][N]: multipliers, 1 / U diagonal,
// U first and second superdiagonal, pivot flags. The recurrences are sequential: one lane
// runs them on the vector's shared-memory copy.
constexpr int kFactorRows = 5;

__global__ void __launch_bounds__(32) k_tri_factor(const double* __restrict__ dg, const double* __restrict__ eg, int N, const double* __restrict__ w, const int* __restrict__ sel,
                                                   double* __restrict__ F, double* __restrict__ Z)
{
  ::trl_detail::pdl_enter();
  extern __shared__ __align__(16) double fs[]; // 5 x N
  const int t = blockIdx.x, lane = threadIdx.x;
  // ||T||_inf (Gershgorin) for the pivot floor
  double nrm = 0.0;
  for (int i = lane; i < N; i += 32) nrm = fmax(nrm, fabs(dg[i]) + (i > 0 ? fabs(eg[i - 1]) : 0.0) + (i + 1 < N ? fabs(eg[i]) : 0.0));
  for (int o = 16; o > 0; o >>= 1) nrm = fmax(nrm, __shfl_xor_sync(0xffffffffu, nrm, o));
  if (!(nrm > 0.0)) nrm = 1.0;
  double* DL = fs;
  double* D = fs + N;
  double* DU = fs + 2 * N;
  double* DU2 = fs + 3 * N;
  double* PV = fs + 4 * N;
  const double lam = w[sel[t]];
  for (int i = lane; i < N; i += 32) {
    D[i] = dg[i] - lam;
    DL[i] = i + 1 < N ? eg[i] : 0.0;
    DU[i] = i + 1 < N ? eg[i] : 0.0;
    DU2[i] = 0.0;
    PV[i] = 0.0;
    Z[static_cast<size_t>(t) * N + i] = hash_unit(static_cast<unsigned>(t), static_cast<unsigned>(i));
  }
  __syncwarp();
  if (lane == 0) {
    const double tiny = DBL_EPSILON * nrm;
    for (int i = 0; i + 1 < N; ++i) {
      if (fabs(D[i]) >= fabs(DL[i])) {
        if (fabs(D[i]) < tiny) D[i] = D[i] < 0.0 ? -tiny : tiny;
        const double fact = DL[i] / D[i];
        DL[i] = fact;
        D[i + 1] -= fact * DU[i];
      }
      else {
        const double fact = D[i] / DL[i];
        D[i] = DL[i];
        DL[i] = fact;
        const double temp = DU[i];
        DU[i] = D[i + 1];
        D[i + 1] = temp - fact * D[i + 1];
        if (i + 2 < N) {
          DU2[i] = DU[i + 1];
          DU[i + 1] = -fact * DU[i + 1];
        }
        PV[i] = 1.0;
      }
    }
    if (fabs(D[N - 1]) < tiny) D[N - 1] = D[N - 1] < 0.0 ? -tiny : tiny;
    for (int i = 0; i < N; ++i) D[i] = 1.0 / D[i];
  }
  __syncwarp();
  for (int idx = lane; idx < kFactorRows * N; idx += 32) F[static_cast<size_t>(t) * kFactorRows * N + idx] = fs[idx];
}

// z_t <- (T - lambda_t I)^{-1} z_t, scaled to unit max-norm
__global__ void __launch_bounds__(32) k_tri_solve(int N, const double* __restrict__ F, double* __restrict__ Z)
{
  ::trl_detail::pdl_enter();
  extern __shared__ __align__(16) double fs[]; // 5 x N factors, N vector
  const int t = blockIdx.x, lane = threadIdx.x;
  for (int idx = lane; idx < kFactorRows * N; idx += 32) fs[idx] = F[static_cast<size_t>(t) * kFactorRows * N + idx];
  double* x = fs + kFactorRows * N;
  for (int i = lane; i < N; i += 32) x[i] = Z[static_cast<size_t>(t) * N + i];
  __syncwarp();
  if (lane == 0) {
    const double* DL = fs;
    const double* RD = fs + N;
    const double* DU = fs + 2 * N;
    const double* DU2 = fs + 3 * N;
    const double* PV = fs + 4 * N;
    double xi = x[0];
    for (int i = 0; i + 1 < N; ++i) { // apply P and L, carrying x[i] in a register
      const double xn = x[i + 1];
      if (PV[i] == 0.0) {
        x[i] = xi;
        xi = xn - DL[i] * xi;
      }
      else {
        x[i] = xn;
        xi = xi - DL[i] * xn;
      }
    }
    x[N - 1] = xi;
    double x1 = x[N - 1] * RD[N - 1]; // x[i+1]
    x[N - 1] = x1;
    double x2 = 0.0; // x[i+2]
    if (N > 1) {
      const double v = (x[N - 2] - DU[N - 2] * x1) * RD[N - 2];
      x[N - 2] = v;
      x2 = x1;
      x1 = v;
    }
    for (int i = N - 3; i >= 0; --i) {
      const double v = (x[i] - DU[i] * x1 - DU2[i] * x2) * RD[i];
      x[i] = v;
      x2 = x1;
      x1 = v;
    }
  }
  __syncwarp();
  double mx = 0.0;
  for (int i = lane; i < N; i += 32) mx = fmax(mx, fabs(x[i]));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const double inv = mx > 0.0 ? 1.0 / mx : 1.0;
  for (int i = lane; i < N; i += 32) Z[static_cast<size_t>(t) * N + i] = x[i] * inv;
}

// classical Gram-Schmidt applied twice, column by column in ascending eigenvalue order, on
// the K vectors held in shared memory (kGlobal: in place in Z, for K x N beyond one CTA's
// shared memory); one CTA of kTriThreads threads
template <bool kGlobal>
__global__ void __launch_bounds__(kTriThreads) k_tri_gs(int N, int K, double* __restrict__ Z)
{
  ::trl_detail::pdl_enter();
  extern __shared__ __align__(16) double zsm[]; // K x N
  double* const zs = kGlobal ? Z : zsm;
  __shared__ double coef[kTriMaxVec];
  __shared__ double red[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = kTriThreads / 32;
  if (!kGlobal) stage(zs, Z, K * N);
  __syncthreads();
  for (int j = 0; j < K; ++j) {
    double* zj = zs + static_cast<size_t>(j) * N;
    for (int pass = 0; pass < 2 && j > 0; ++pass) {
      for (int i = warp; i < j; i += NW) {
        const double* zi = zs + static_cast<size_t>(i) * N;
        double s = 0.0;
        for (int n = lane; n < N; n += 32) s = fma(zi[n], zj[n], s);
        s = warp_sum(s);
        if (lane == 0) coef[i] = s;
      }
      __syncthreads();
      for (int n = tid; n < N; n += kTriThreads) {
        double v = zj[n];
        for (int i = 0; i < j; ++i) v = fma(-coef[i], zs[static_cast<size_t>(i) * N + n], v);
        zj[n] = v;
      }
      __syncthreads();
    }
    double s = 0.0;
    for (int n = tid; n < N; n += kTriThreads) s = fma(zj[n], zj[n], s);
    s = block_sum(s, red);
    const double inv = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    for (int n = tid; n < N; n += kTriThreads) zj[n] *= inv;
    __syncthreads();
  }
  if (!kGlobal)
    for (int idx = tid; idx < K * N; idx += kTriThreads) Z[idx] = zs[idx];
}

// Back-transform X = Q Z, Q = H_0 ... H_{N-3}, in chunks of kWyRows reflectors: a chunk
// H_a ... H_b equals I - V T V^T (compact WY form, T upper triangular: T_ii = tau_i,
// T[0:i, i] = -tau_i T[0:i, 0:i] V[:, 0:i]^T v_i), so a chunk is three small matrix
// products on the vectors instead of kWyRows dependent reflector applications.
constexpr int kWyRows = 16;
constexpr int kWyVecs = 1; // vectors per CTA: the chunk products are latency-bound, so one vector per CTA spreads them over K SMs

// T of chunk c (reflectors c * kWyRows ...) into Tw[c][kWyRows][kWyRows]
__global__ void __launch_bounds__(256) k_wy_factor(const double* __restrict__ refl, const double* __restrict__ tau, int N, double* __restrict__ Tw)
{
  ::trl_detail::pdl_enter();
  extern __shared__ __align__(16) double vs[]; // kWyRows x N
  __shared__ double G[kWyRows][kWyRows], Tt[kWyRows][kWyRows];
  const int R = N - 2;
  const int k0 = blockIdx.x * kWyRows;
  const int b = R - k0 < kWyRows ? R - k0 : kWyRows;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  stage(vs, refl + static_cast<size_t>(k0) * N, b * N);
  __syncthreads();
  for (int rr = 0; rr < b; ++rr) // v_k is zero up to row k (refl holds nothing there)
    for (int i = tid; i <= k0 + rr; i += blockDim.x) vs[rr * N + i] = 0.0;
  __syncthreads();
  for (int pq = warp; pq < b * b; pq += blockDim.x >> 5) {
    const int p = pq / b, q = pq % b;
    if (p >= q) continue; // strictly upper part: G[p][q] = v_p . v_q
    double s = 0.0;
    for (int i = lane; i < N; i += 32) s = fma(vs[p * N + i], vs[q * N + i], s);
    s = warp_sum(s);
    if (lane == 0) G[p][q] = s;
  }
  __syncthreads();
  if (warp == 0) {
    for (int i = 0; i < b; ++i) {
      const double ti = tau[k0 + i];
      // lane j < i: T[j][i] = -tau_i sum_{m=j}^{i-1} T[j][m] G[m][i]
      double v = 0.0;
      if (lane < i) {
        for (int m = lane; m < i; ++m) v = fma(Tt[lane][m], G[m][i], v);
        v = -ti * v;
      }
      __syncwarp();
      if (lane < i) Tt[lane][i] = v;
      if (lane == i) Tt[i][i] = ti;
      if (lane > i && lane < kWyRows) Tt[lane][i] = 0.0;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int e = tid; e < kWyRows * kWyRows; e += blockDim.x) {
    const int p = e / kWyRows, q = e % kWyRows;
    Tw[static_cast<size_t>(blockIdx.x) * kWyRows * kWyRows + e] = (p < b && q < b) ? Tt[p][q] : 0.0;
  }
}

__global__ void __launch_bounds__(256) k_backtransform(const double* __restrict__ Z, int K, int N, const double* __restrict__ refl, const double* __restrict__ Tw,
                                                       double* __restrict__ X)
{
  ::trl_detail::pdl_enter();
  extern __shared__ __align__(16) double sm[]; // kWyRows x N reflectors | kWyVecs x N vectors
  double* vs = sm;
  double* xs = sm + kWyRows * N;
  __shared__ double W[kWyRows][kWyVecs], W2[kWyRows][kWyVecs], Ts[kWyRows][kWyRows];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t0 = blockIdx.x * kWyVecs;
  const int nv = K - t0 < kWyVecs ? K - t0 : kWyVecs;
  stage(xs, Z + static_cast<size_t>(t0) * N, nv * N);
  const int R = N - 2;
  const int nch = (R + kWyRows - 1) / kWyRows;
  for (int c = nch - 1; c >= 0; --c) {
    const int k0 = c * kWyRows;
    const int b = R - k0 < kWyRows ? R - k0 : kWyRows;
    __syncthreads(); // previous chunk done with vs, Ts, W2
    stage(vs, refl + static_cast<size_t>(k0) * N, b * N);
    for (int e = tid; e < kWyRows * kWyRows; e += blockDim.x) Ts[e / kWyRows][e % kWyRows] = Tw[static_cast<size_t>(c) * kWyRows * kWyRows + e];
    __syncthreads();
    for (int rr = 0; rr < b; ++rr) // v_k is zero up to row k (refl holds nothing there)
      for (int i = tid; i <= k0 + rr; i += blockDim.x) vs[rr * N + i] = 0.0;
    __syncthreads();
    // W = V^T X: warp per (row, vector) pair
    for (int pv = warp; pv < b * nv; pv += blockDim.x >> 5) {
      const int rr = pv / nv, v = pv % nv;
      double s0 = 0.0, s1 = 0.0;
      int i = lane;
      for (; i + 32 < N; i += 64) {
        s0 = fma(vs[rr * N + i], xs[v * N + i], s0);
        s1 = fma(vs[rr * N + i + 32], xs[v * N + i + 32], s1);
      }
      if (i < N) s0 = fma(vs[rr * N + i], xs[v * N + i], s0);
      const double s = warp_sum(s0 + s1);
      if (lane == 0) W[rr][v] = s;
    }
    __syncthreads();
    if (tid < b * nv) { // W2 = T W
      const int rr = tid / nv, v = tid % nv;
      double s = 0.0;
      for (int m = rr; m < b; ++m) s = fma(Ts[rr][m], W[m][v], s);
      W2[rr][v] = s;
    }
    __syncthreads();
    for (int idx = tid; idx < nv * N; idx += blockDim.x) { // X -= V W2
      const int v = idx / N, i = idx % N;
      double x = xs[idx];
      for (int rr = 0; rr < b; ++rr) x = fma(-vs[rr * N + i], W2[rr][v], x);
      xs[idx] = x;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nv * N; idx += blockDim.x) X[static_cast<size_t>(t0) * N + idx] = xs[idx];
}

// selected ascending indices: sel[t] (ascending), slot[c] = t for rank c < K
__global__ void k_select(const int* __restrict__ perm, int K, int* __restrict__ sel, int* __restrict__ slot)
{
  ::trl_detail::pdl_enter();
  const int c = threadIdx.x;
  if (c >= K) return;
  const int a = perm[c];
  int t = 0;
  for (int q = 0; q < K; ++q) t += perm[q] < a;
  sel[t] = a;
  slot[c] = t;
}

// Y in block layout: column c < K is X[slot[c]], the rest zero
__global__ void k_scatter_partial(const double* __restrict__ X, const int* __restrict__ slot, int nblk, int bs, int K, double* __restrict__ Y)
{
  ::trl_detail::pdl_enter();
  const int N = nblk * bs;
  const int64_t total = static_cast<int64_t>(N) * N;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int cj = static_cast<int>(e % bs);
    const int64_t q = e / bs;
    const int ri = static_cast<int>(q % bs);
    const int64_t blk = q / bs;
    const int bj = static_cast<int>(blk % nblk), bi = static_cast<int>(blk / nblk);
    const int row = bi * bs + ri, col = bj * bs + cj;
    Y[e] = col < K ? X[static_cast<int64_t>(slot[col]) * N + row] : 0.0;
  }
}

__global__ void k_count_partial(const double* __restrict__ X, const int* __restrict__ slot, const double* __restrict__ evals_sorted, const double* __restrict__ beta, int nblk, int bs,
                                int ncheck, double tol, int* __restrict__ count)
{
  ::trl_detail::pdl_enter();
  const int N = nblk * bs;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncheck; c += gridDim.x * blockDim.x) {
    const double* y = X + static_cast<int64_t>(slot[c]) * N + (nblk - 1) * bs;
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

// zero the block-layout columns >= K of Y
__global__ void k_zero_cols(double* __restrict__ Y, int nblk, int bs, int K)
{
  ::trl_detail::pdl_enter();
  const int N = nblk * bs;
  const int64_t total = static_cast<int64_t>(N) * N;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int cj = static_cast<int>(e % bs);
    const int bj = static_cast<int>((e / (static_cast<int64_t>(bs) * bs)) % nblk);
    if (bj * bs + cj >= K) Y[e] = 0.0;
  }
}

using TriKernel = void (*)(double*, int, double*, double*, double*, double*);

struct TriVariant {
  TriKernel fn;
  int C;       // CTAs in the cluster
  bool global; // rows in global memory
  int max_n;
};

constexpr TriVariant kTriVariants[] = {
    {k_tridiag<8, false>, 8, false, kTriMaxN8},
    {k_tridiag<16, false>, 16, false, kTriMaxN16},
    {k_tridiag<16, true>, 16, true, kTriMaxN},
    {k_tridiag<8, true>, 8, true, kTriMaxN},
};
constexpr int kNumTriVariants = sizeof(kTriVariants) / sizeof(kTriVariants[0]);

void tri_config(const TriVariant& v, int N, cudaStream_t stream, cudaLaunchConfig_t& cfg, cudaLaunchAttribute& attr)
{
  cfg = cudaLaunchConfig_t{};
  cfg.gridDim = dim3(v.C);
  cfg.blockDim = dim3(kTriThreads);
  cfg.dynamicSmemBytes = tridiag_smem(N, v.C, v.global);
  cfg.stream = stream;
  attr = cudaLaunchAttribute{};
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = v.C;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
}

// The first variant that takes N and can be resident on `device`, or null. Checked once per
// device: function attributes belong to the current device.
const TriVariant* tri_variant(int device, int N)
{
  static int ok[64][kNumTriVariants];
  static bool checked[64];
  static std::mutex lock;
  std::lock_guard<std::mutex> g(lock);
  if (!checked[device]) {
    checked[device] = true;
    const bool common = cudaFuncSetAttribute(k_tri_gs<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kTriGsMaxBytes)) == cudaSuccess &&
                        cudaFuncSetAttribute(k_tri_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sizeof(double) * (kFactorRows + 1) * kTriMaxN)) == cudaSuccess &&
                        cudaFuncSetAttribute(k_tri_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sizeof(double) * kFactorRows * kTriMaxN)) == cudaSuccess &&
                        cudaFuncSetAttribute(k_backtransform, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sizeof(double) * (kWyRows + kWyVecs) * kTriMaxN)) == cudaSuccess &&
                        cudaFuncSetAttribute(k_wy_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sizeof(double) * kWyRows * kTriMaxN)) == cudaSuccess;
    for (int i = 0; i < kNumTriVariants && common; ++i) {
      const TriVariant& v = kTriVariants[i];
      if (cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(tridiag_smem(v.max_n, v.C, v.global))) != cudaSuccess) continue;
      if (v.C > 8 && cudaFuncSetAttribute(v.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) continue;
      cudaLaunchConfig_t cfg{};
      cudaLaunchAttribute attr{};
      tri_config(v, v.max_n, nullptr, cfg, attr);
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, v.fn, &cfg) == cudaSuccess && clusters > 0) ok[device][i] = 1;
    }
    cudaGetLastError();
  }
  for (int i = 0; i < kNumTriVariants; ++i)
    if (ok[device][i] && N <= kTriVariants[i].max_n) return &kTriVariants[i];
  return nullptr;
}

} // namespace

extern "C" int trl_cuda_small_eigen_partial(trl_cuda_handle h, const double* T, int nblk, int bs, const double* beta, int nev, double tol, int kvec, double* evals, double* evecs,
                                            double* host_evals, int* host_nconv)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || nblk <= 0 || !T || !beta || !evals || !evecs || !host_evals || !host_nconv) return set_error(h, TRL_EINVAL, "bad small_eigen arguments");
  const int N = nblk * bs;
  if (kvec < 0 || kvec > N) return set_error(h, TRL_EINVAL, "kvec %d outside [0, %d]", kvec, N);
  if (h->device < 0 || h->device >= 64) return set_error(h, TRL_EINVAL, "device index %d", h->device);
  const TriVariant* tv = tri_variant(h->device, N);
  if (N < 3 || kvec > kTriMaxVec || !tv) {
    if (int st = trl_cuda_small_eigen(h, T, nblk, bs, beta, nev, tol, evals, evecs, host_evals, host_nconv)) return st;
    launch(k_zero_cols, grid_for(h, static_cast<int64_t>(N) * N, 256, 4), 256, 0, h->stream, evecs, nblk, bs, kvec);
    return after_launch(h, "zero columns");
  }
  ProfScope prof(h, PROF_SMALL_EIGEN, 16.0 * N * N);
  const int K = kvec > 0 ? kvec : 1;
  // workspace: A (N*N) | refl (N*N) | d | e | tau | w (N each) | Z (N*K) | X (N*K) |
  // factors (5 N*K) | perm, sel, slot (N ints each) | zero flag, count
  const size_t NN = static_cast<size_t>(N) * N, NK = static_cast<size_t>(N) * K;
  const size_t nchunks = static_cast<size_t>(N - 2 + kWyRows - 1) / kWyRows;
  const size_t doubles = 2 * NN + 4 * static_cast<size_t>(N) + (2 + kFactorRows) * NK + nchunks * kWyRows * kWyRows;
  const size_t ints = 3 * static_cast<size_t>(N) + 8;
  char* ws = static_cast<char*>(workspace(h, sizeof(double) * (doubles + 1) + sizeof(int) * ints + 256));
  if (!ws) return TRL_ENOMEM;
  double* A = reinterpret_cast<double*>(ws);
  double* refl = A + NN;
  double* d = refl + NN;
  double* e = d + N;
  double* tau = e + N;
  double* w = tau + N;
  double* Z = w + N;
  double* X = Z + NK;
  double* F = X + NK;
  double* Tw = F + kFactorRows * NK;
  int* perm = reinterpret_cast<int*>(Tw + nchunks * kWyRows * kWyRows);
  int* sel = perm + N;
  int* slot = sel + N;
  int* flags = slot + N; // [0] = 0 (no solver error), [1] = converged count
  double* tmax = reinterpret_cast<double*>(ws + (sizeof(double) * doubles + sizeof(int) * ints + 15) / 16 * 16);

  const unsigned g = grid_for(h, static_cast<int64_t>(N) * N, 256, 4);
  launch(k_max_abs, 1, 1024, 0, h->stream, T, static_cast<int64_t>(N) * N, tmax);
  launch(k_assemble_dense, g, 256, 0, h->stream, T, nblk, bs, tmax, A);
  if (int st = after_launch(h, "assemble")) return st;
  cudaMemsetAsync(flags, 0, 2 * sizeof(int), h->stream);
  {
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr{};
    tri_config(*tv, N, h->stream, cfg, attr);
    cudaLaunchKernelEx(&cfg, tv->fn, A, N, d, e, tau, refl);
    if (int st = after_launch(h, "tridiagonalise")) return st;
  }
  launch(k_bisect, (N + 7) / 8, 256, 0, h->stream, d, e, N, w);
  if (int st = after_launch(h, "bisect")) return st;
  launch(k_rank, (N + 255) / 256, 256, 0, h->stream, w, N, perm, evals, flags, h->d_status);
  if (int st = after_launch(h, "rank")) return st;
  launch(k_select, 1, kTriMaxVec, 0, h->stream, perm, K, sel, slot);
  if (int st = after_launch(h, "select")) return st;
  launch(k_tri_factor, K, 32, sizeof(double) * kFactorRows * N, h->stream, d, e, N, w, sel, F, Z);
  if (int st = after_launch(h, "tridiagonal factor")) return st;
  for (int it = 0; it < kTriIters; ++it) {
    launch(k_tri_solve, K, 32, sizeof(double) * (kFactorRows + 1) * N, h->stream, N, F, Z);
    if (int st = after_launch(h, "inverse iteration")) return st;
  }
  if (sizeof(double) * NK > kTriGsMaxBytes) launch(k_tri_gs<true>, 1, kTriThreads, 0, h->stream, N, K, Z);
  else launch(k_tri_gs<false>, 1, kTriThreads, sizeof(double) * NK, h->stream, N, K, Z);
  if (int st = after_launch(h, "gram-schmidt")) return st;
  const int nch = (N - 2 + kWyRows - 1) / kWyRows;
  launch(k_wy_factor, nch, 256, sizeof(double) * kWyRows * N, h->stream, refl, tau, N, Tw);
  if (int st = after_launch(h, "wy factor")) return st;
  launch(k_backtransform, (K + kWyVecs - 1) / kWyVecs, 256, sizeof(double) * (kWyRows + kWyVecs) * N, h->stream, Z, K, N, refl, Tw, X);
  if (int st = after_launch(h, "back-transform")) return st;
  launch(k_scatter_partial, g, 256, 0, h->stream, X, slot, nblk, bs, kvec, evecs);
  if (int st = after_launch(h, "scatter")) return st;
  const int ncheck = nev < kvec ? nev : kvec;
  if (ncheck > 0) {
    launch(k_count_partial, (ncheck + 127) / 128, 128, 0, h->stream, X, slot, evals, beta, nblk, bs, ncheck, tol, flags + 1);
    if (int st = after_launch(h, "count")) return st;
  }
  const size_t w_bytes = sizeof(double) * N;
  char* pin = static_cast<char*>(pinned(h, w_bytes + 64));
  if (!pin) return TRL_ENOMEM;
  cudaMemcpyAsync(pin, evals, w_bytes, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(pin + w_bytes, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  int st = trl_cuda_synchronize(h);
  if (st) return st;
  std::memcpy(host_evals, pin, w_bytes);
  std::memcpy(host_nconv, pin + w_bytes, sizeof(int));
  return TRL_OK;
}
