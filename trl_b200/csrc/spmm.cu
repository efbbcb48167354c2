// CSR sparse operator against a row-major block: Y = alpha*A*X + beta*X, and the SDDMM
// used by the eigenvalue adjoint.
//
// SpMM scheduling: a row is owned by a group of LPR lanes; each lane carries VEC adjacent
// columns of the block so that one X row is gathered with LPR 16-byte loads. A warp's
// consecutive rows form one contiguous CSR range, staged in shared memory with coalesced
// loads, so that every X gather is issued without waiting on index loads of the other
// entries (see k_spmm). Accumulation is in the storage type (FP32 for the mixed mode, as
// the FP32 SpMM is specified; FP64 otherwise).
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

using namespace trl_detail;

constexpr int kThreads = 256;

template <typename T, int BS>
struct SpmmShape {
  static constexpr int max_vec = 16 / static_cast<int>(sizeof(T));
  static constexpr int VEC = max_vec < BS ? max_vec : BS;
  static constexpr int LPR = BS / VEC;                   // lanes per row: 1..8
  static constexpr int RPW = 32 / LPR;                   // rows per warp iteration
  static constexpr int CH = RPW * 8 > 64 ? RPW * 8 : 64; // (col, val) pairs staged per warp per chunk
  static constexpr int PF = CH / 32;                     // pairs each lane stages per chunk
  // Measured on B200 (96^3 7-point operator, block 8): FP64 4 gathers in flight per lane
  // and 6 CTAs per SM (40 registers) take 49.6 us against 53.4 us for 8 gathers at 4 CTAs
  // per SM; FP32 prefers 8 gathers at 4 CTAs per SM (28.8 us). A software prefetch of the
  // next row group's CSR range, and contiguous row ranges per CTA, measured slower.
  static constexpr int UG = sizeof(T) == 8 ? 4 : 8;      // gathers a lane issues before its FMAs
  static constexpr int MINB = sizeof(T) == 8 ? 6 : 4;    // CTAs per SM the registers must allow
};

// A row of a warp iteration is swept by all the warp's row groups together when it holds
// more than kLongRow entries and more than twice the iteration's mean row length: the
// per-row walk keeps every group busy for the longest row's length, which on a Zipf row-length
// pattern (median 21, p99 326) leaves 70% of the lane slots idle.
constexpr int kLongRow = 32;

// A warp owns RPW consecutive rows per iteration; within it a group of LPR lanes owns a row
// and each lane VEC adjacent columns of the block.
//  1. rowptr of the warp's rows is loaded one iteration ahead;
//  2. the rows' (col, val) pairs - one contiguous CSR range - are staged in shared memory
//     with coalesced warp-wide loads, CH pairs at a time;
//  3. each group walks its row's pairs in the stage and issues UG independent X gathers
//     (16 bytes per lane) before the FMAs that consume them;
//  4. long rows (kLongRow) are left out of step 3 and swept afterwards, one at a time, by
//     all groups (group g takes every RPW-th pair from g), then summed over the groups
//     with butterfly shuffles. Chunks that hold only long-row pairs are not staged in step 2.
//  With MB (several blocks), a range that fits one stage is staged once for all blocks and
//  walked per row.
template <typename T, int BS, bool MB>
__global__ void __launch_bounds__(kThreads, SpmmShape<T, BS>::MINB) k_spmm(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind,
                                                                         const T* __restrict__ vals, const T* __restrict__ X, T* Y, T alpha, T beta, T gamma,
                                                                         const T* W, int nb, int64_t bstride)
{
  ::trl_detail::pdl_enter();
  using S = SpmmShape<T, BS>;
  constexpr int VEC = S::VEC, LPR = S::LPR, RPW = S::RPW, UG = S::UG, CH = S::CH, PF = S::PF;
  constexpr int WPC = kThreads / 32;
  // The multi-block walk and FP64 with one column per lane have no registers left for the
  // long-row sweep under the 6-CTA bound (ptxas spills them); they walk every row per row.
  constexpr bool COOP = !MB && !(sizeof(T) == 8 && BS == 1);
  __shared__ int s_col[WPC][CH];
  __shared__ T s_val[WPC][CH];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int sub = lane % LPR;
  const int grp = lane / LPR;
  const int64_t step = static_cast<int64_t>(gridDim.x) * WPC * RPW;
  int64_t rbase = (static_cast<int64_t>(blockIdx.x) * WPC + w) * RPW;
  if (rbase >= n) return; // whole warp
  // lane l < RPW holds rowptr[row l], every lane the end offset rowptr[row RPW] (rows past
  // n read rowptr[n]: empty rows); iterations past n are empty
  auto load_rp = [&](int64_t base, int& rp, int& rpe) {
    rp = (base < n && lane < RPW) ? __ldg(rowptr + min(base + lane, n)) : 0;
    rpe = (base < n) ? __ldg(rowptr + min(base + RPW, n)) : 0;
  };
  int rp0, rpe0;
  load_rp(rbase, rp0, rpe0);

  for (; rbase < n; rbase += step) {
    int rp1, rpe1;
    load_rp(rbase + step, rp1, rpe1);
    const int s = __shfl_sync(0xffffffffu, rp0, 0);
    const int e = rpe0;
    const int kb = __shfl_sync(0xffffffffu, rp0, grp);
    const int kn = __shfl_sync(0xffffffffu, rp0, (grp + 1) & 31);
    const int ke = (grp + 1 == RPW) ? rpe0 : kn;
    // The CSR range is staged once when it fits the stage and then applied to every block
    // (X, Y, W hold nb blocks bstride elements apart); longer ranges are staged chunk by
    // chunk for each block.
    const bool one_chunk = MB && (e - s) <= CH; // uniform over the warp
    // Each group tests its own row (len * RPW > 2 (e - s), without overflow); bit g * LPR of
    // `longs` marks row g. No shuffle: the walk is bound by the shared-memory/L1 pipe, where
    // one more shuffle per iteration cost the stencil 4%.
    const int len = ke - kb;
    const bool mine_long = COOP && !one_chunk && len > kLongRow && static_cast<unsigned>(len) > static_cast<unsigned>(e - s) / (RPW / 2);
    const unsigned longs = COOP ? __ballot_sync(0xffffffffu, mine_long && sub == 0) : 0u;
    const int kw = mine_long ? kb : ke; // end of this group's per-row walk
    auto stage = [&](int cs, int end) {
#pragma unroll
      for (int q = 0; q < PF; ++q) {
        const int p = cs + q * 32 + lane;
        if (p < end) {
          s_col[w][q * 32 + lane] = ld_stream(colind + p);
          s_val[w][q * 32 + lane] = ld_stream(vals + p);
        }
      }
      __syncwarp();
    };
    if (one_chunk) stage(s, e);
    for (int b = 0; b < (MB ? nb : 1); ++b) {
      const T* Xb = X + static_cast<int64_t>(b) * bstride;
      T acc[VEC];
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[i] = T(0);
      for (int cs = s; cs < e; cs += CH) {
        const int lo = max(kb, cs) - cs, hi = min(kw, cs + CH) - cs;
        if (longs != 0 && !__any_sync(0xffffffffu, lo < hi)) continue; // only long-row pairs
        if (!one_chunk) stage(cs, e);
        for (int t = lo; t < hi; t += UG) {
          T x[UG][VEC];
          T wv[UG];
#pragma unroll
          for (int u = 0; u < UG; ++u) {
            if (t + u < hi) {
              wv[u] = s_val[w][t + u];
              load_vec<T, VEC>(Xb + static_cast<int64_t>(s_col[w][t + u]) * BS + sub * VEC, x[u]);
            }
            else {
              wv[u] = T(0);
#pragma unroll
              for (int i = 0; i < VEC; ++i) x[u][i] = T(0);
            }
          }
#pragma unroll
          for (int u = 0; u < UG; ++u)
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = fma(wv[u], x[u][i], acc[i]);
        }
        if (!one_chunk) __syncwarp(); // the stage is rewritten by the next chunk
      }

      for (unsigned m = longs; m != 0; m &= m - 1) { // warp-uniform
        const int r = (__ffs(m) - 1) / LPR; // the row, and the group that writes it
        const int rb = __shfl_sync(0xffffffffu, kb, r * LPR);
        const int re = __shfl_sync(0xffffffffu, ke, r * LPR);
        T lacc[VEC];
#pragma unroll
        for (int i = 0; i < VEC; ++i) lacc[i] = T(0);
        for (int cs = rb; cs < re; cs += CH) {
          stage(cs, re);
          const int cnt = min(re - cs, CH);
          for (int t = grp; t < cnt; t += RPW * UG) {
            T x[UG][VEC];
            T wv[UG];
#pragma unroll
            for (int u = 0; u < UG; ++u) {
              const int tu = t + u * RPW;
              if (tu < cnt) {
                wv[u] = s_val[w][tu];
                load_vec<T, VEC>(Xb + static_cast<int64_t>(s_col[w][tu]) * BS + sub * VEC, x[u]);
              }
              else {
                wv[u] = T(0);
#pragma unroll
                for (int i = 0; i < VEC; ++i) x[u][i] = T(0);
              }
            }
#pragma unroll
            for (int u = 0; u < UG; ++u)
#pragma unroll
              for (int i = 0; i < VEC; ++i) lacc[i] = fma(wv[u], x[u][i], lacc[i]);
          }
          __syncwarp(); // the stage is rewritten by the next chunk
        }
        // lane = grp * LPR + sub: sum over the group bits
#pragma unroll
        for (int off = LPR; off < 32; off <<= 1)
#pragma unroll
          for (int i = 0; i < VEC; ++i) lacc[i] += __shfl_xor_sync(0xffffffffu, lacc[i], off);
        if (grp == r) {
#pragma unroll
          for (int i = 0; i < VEC; ++i) acc[i] = lacc[i];
        }
      }

      const int64_t row = rbase + grp;
      if (row < n) {
        T* Yb = Y + static_cast<int64_t>(b) * bstride;
        T y[VEC];
        if (beta != T(0)) {
          T x[VEC];
          load_vec<T, VEC>(Xb + row * BS + sub * VEC, x);
#pragma unroll
          for (int i = 0; i < VEC; ++i) y[i] = fma(alpha, acc[i], beta * x[i]); // explicit: the same rounding as the sliced-ELL kernel
        }
        else {
#pragma unroll
          for (int i = 0; i < VEC; ++i) y[i] = alpha * acc[i];
        }
        if (W) { // W may be Y itself: this lane reads its values before it writes them
          const T* Wb = W + static_cast<int64_t>(b) * bstride;
          T wv[VEC];
#pragma unroll
          for (int i = 0; i < VEC; ++i) wv[i] = Wb[row * BS + sub * VEC + i];
#pragma unroll
          for (int i = 0; i < VEC; ++i) y[i] = fma(gamma, wv[i], y[i]);
        }
        store_vec<T, VEC>(Yb + row * BS + sub * VEC, y);
      }
    }
    if (one_chunk) __syncwarp(); // the stage is rewritten by the next iteration
    rp0 = rp1;
    rpe0 = rpe1;
  }
}

// out[p] = sum_c w[c] X[row(p), c] X[col(p), c]; one warp per row, lanes over its entries.
__global__ void __launch_bounds__(kThreads) k_sddmm(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind, const double* __restrict__ X, int k,
                                                    const double* __restrict__ w, double* __restrict__ out)
{
  ::trl_detail::pdl_enter();
  const int lane = threadIdx.x & 31;
  const int64_t warp_global = static_cast<int64_t>(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
  const int64_t warp_stride = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  for (int64_t row = warp_global; row < n; row += warp_stride) {
    const int kbeg = __ldg(rowptr + row), kend = __ldg(rowptr + row + 1);
    const double* xr = X + row * k;
    for (int p = kbeg + lane; p < kend; p += 32) {
      const double* xc = X + static_cast<int64_t>(__ldg(colind + p)) * k;
      double s = 0.0;
      for (int c = 0; c < k; ++c) s = fma(__ldg(w + c) * __ldg(xr + c), __ldg(xc + c), s);
      out[p] = s;
    }
  }
}

} // namespace

using namespace trl_detail;

extern "C" {

static int spmm_impl(trl_cuda_context* h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, int nb, double alpha, double beta, double gamma,
                     const void* W)
{
  if (nb < 1) return set_error(h, TRL_EINVAL, "block count %d", nb);
  if (!A || !X || !Y) return set_error(h, TRL_EINVAL, "null pointer");
  if (!valid_dtype(dtype) || A->value_dtype != dtype) return set_error(h, TRL_ENOTSUP, "SpMM needs CSR values and block in the same dtype (got %d and %d)", A->value_dtype, dtype);
  if (!valid_bs(bs)) return set_error(h, TRL_ENOTSUP, "unsupported block size %d", bs);
  if (A->n < 0 || A->nnz < 0 || A->nnz >= (int64_t(1) << 31)) return set_error(h, TRL_EINVAL, "bad CSR sizes");
  if (A->n == 0) return TRL_OK;
  if (!A->rowptr || (A->nnz > 0 && (!A->colind || !A->values))) return set_error(h, TRL_EINVAL, "null CSR array");
  const size_t es = dtype == TRL_F64 ? 8 : 4;
  const auto overlap = [&](const void* a, const void* b) {
    const auto pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = static_cast<uintptr_t>(nb) * A->n * bs * es;
    return pa < pb + len && pb < pa + len;
  };
  if (overlap(X, Y) || (W && overlap(W, X)) || (W && W != Y && overlap(W, Y)))
    return set_error(h, TRL_EINVAL, "SpMM input must overlap neither output nor third operand");
  if (((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) % (es * bs < 16 ? es * bs : 16)) != 0)
    return set_error(h, TRL_EINVAL, "block vectors must be aligned to min(16, bs*elem) bytes");
  ProfScope prof(h, PROF_SPMM, A->nnz * (es + 4.0) + 4.0 * (A->n + 1) + nb * (W ? 3.0 : 2.0) * A->n * bs * es, 2.0 * A->nnz * bs * nb);
  int st = TRL_OK;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, {
    using S = SpmmShape<T, BS>;
    // one resident wave: every warp strides over the rows (its rowptr prefetch pays off)
    const auto run = [&](auto kernel) {
      static int resident = 0; // one per instantiation of the kernel
      if (resident == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kThreads, 0) != cudaSuccess || resident < 1) resident = S::MINB;
        cudaGetLastError();
      }
      const unsigned grid = grid_for(h, (A->n + S::RPW - 1) / S::RPW, kThreads / 32, resident);
      trl_detail::launch(kernel, grid, kThreads, 0, h->stream, A->n, A->rowptr, A->colind, static_cast<const T*>(A->values), static_cast<const T*>(X), static_cast<T*>(Y),
                                               static_cast<T>(alpha), static_cast<T>(beta), static_cast<T>(gamma), static_cast<const T*>(W), nb, A->n * BS);
    };
    if (nb > 1) run(k_spmm<T, BS, true>);
    else run(k_spmm<T, BS, false>);
    st = after_launch(h, "spmm");
  }));
  return st;
}

int trl_cuda_spmm(trl_cuda_handle h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, double alpha, double beta)
{
  TRL_CHECK_HANDLE(h);
  return spmm_impl(h, A, dtype, X, Y, bs, 1, alpha, beta, 0.0, nullptr);
}

int trl_cuda_spmm3(trl_cuda_handle h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, double alpha, double beta, double gamma, const void* W)
{
  TRL_CHECK_HANDLE(h);
  return spmm_impl(h, A, dtype, X, Y, bs, 1, alpha, beta, gamma, W);
}

int trl_cuda_spmm_blocks(trl_cuda_handle h, const trl_csr* A, int dtype, const void* X, void* Y, int bs, int nb, double alpha, double beta, double gamma, const void* W)
{
  TRL_CHECK_HANDLE(h);
  return spmm_impl(h, A, dtype, X, Y, bs, nb, alpha, beta, gamma, W);
}

int trl_cuda_sddmm(trl_cuda_handle h, const trl_csr* P, const double* X, int k, const double* w, double* out)
{
  TRL_CHECK_HANDLE(h);
  if (!P || !X || !w || !out) return set_error(h, TRL_EINVAL, "null pointer");
  if (k <= 0) return set_error(h, TRL_EINVAL, "k must be positive");
  if (P->n == 0 || P->nnz == 0) return TRL_OK;
  ProfScope prof(h, PROF_SDDMM, 12.0 * P->nnz + 4.0 * (P->n + 1) + 8.0 * P->n * k, 3.0 * P->nnz * k);
  const unsigned grid = grid_for(h, P->n, kThreads / 32, 16);
  launch(k_sddmm, grid, kThreads, 0, h->stream, P->n, P->rowptr, P->colind, X, k, w, out);
  return after_launch(h, "sddmm");
}

int trl_cuda_eigen_adjoint(trl_cuda_handle h, const trl_csr* P, const double* X, int k, const double* host_evals, const double* host_weights, double cluster_rtol, int kind,
                           double* grad)
{
  TRL_CHECK_HANDLE(h);
  if (!P || !X || !host_evals || !host_weights || !grad) return set_error(h, TRL_EINVAL, "null pointer");
  if (k <= 0 || k > 4096) return set_error(h, TRL_EINVAL, "k must be in [1, 4096]");
  if (kind != 0 && kind != 1) return set_error(h, TRL_EINVAL, "kind must be 0 (operator) or 1 (mass)");
  if (cluster_rtol < 0.0) return set_error(h, TRL_EINVAL, "negative cluster tolerance");
  // cluster-averaged coefficients (host; k is small). Eigenvalues are grouped by sorting and
  // joining neighbours closer than cluster_rtol * max|lambda|.
  std::vector<double> c(k);
  std::vector<int> order(k);
  double amax = 0.0;
  for (int i = 0; i < k; ++i) {
    order[i] = i;
    amax = std::fmax(amax, std::fabs(host_evals[i]));
  }
  std::sort(order.begin(), order.end(), [&](int a, int b) { return host_evals[a] < host_evals[b]; });
  const double gap = cluster_rtol * amax;
  for (int s = 0; s < k;) {
    int e = s + 1;
    while (e < k && host_evals[order[e]] - host_evals[order[e - 1]] <= gap) ++e;
    double mean = 0.0;
    for (int q = s; q < e; ++q) mean += host_weights[order[q]];
    mean /= (e - s);
    for (int q = s; q < e; ++q) {
      const int i = order[q];
      c[i] = kind == 0 ? mean : -mean * host_evals[i];
    }
    s = e;
  }
  double* dc = static_cast<double*>(workspace2(h, sizeof(double) * k));
  if (!dc) return TRL_ENOMEM;
  if (int st = trl_cuda_memcpy(h, dc, c.data(), sizeof(double) * k, TRL_H2D)) return st;
  if (int st = trl_cuda_sddmm(h, P, X, k, dc, grad)) return st;
  // the host coefficient array goes out of scope: make sure the copy has been consumed
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "eigen_adjoint: %s", cudaGetErrorString(e));
  return TRL_OK;
}

} // extern "C"

namespace {

__global__ void __launch_bounds__(256) k_norm1(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind, const void* __restrict__ vals, int f64,
                                               double alpha, double beta, unsigned long long* __restrict__ out)
{
  ::trl_detail::pdl_enter();
  double best = 0.0;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    bool diag = false;
    for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) {
      const double a = f64 ? static_cast<const double*>(vals)[p] : static_cast<double>(static_cast<const float*>(vals)[p]);
      if (colind[p] == r) {
        s += fabs(alpha * a + beta);
        diag = true;
      }
      else
        s += fabs(alpha * a);
    }
    if (!diag) s += fabs(beta);
    best = fmax(best, s);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(best)));
}

// Monotone map of doubles onto unsigned 64-bit integers (for atomicMin/atomicMax).
__device__ __forceinline__ unsigned long long ordered_bits(double x)
{
  const unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(x));
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

// Gershgorin interval of alpha*A + beta*I: [min_i (c_i - r_i), max_i (c_i + r_i)] with
// c_i = alpha*a_ii + beta and r_i = |alpha| * sum_{j != i} |a_ij|.
__global__ void __launch_bounds__(256) k_gershgorin(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind, const void* __restrict__ vals,
                                                    int f64, double alpha, double beta, unsigned long long* __restrict__ lo_hi)
{
  ::trl_detail::pdl_enter();
  double lo = INFINITY, hi = -INFINITY;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double c = beta, rad = 0.0;
    for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) {
      const double a = f64 ? static_cast<const double*>(vals)[p] : static_cast<double>(static_cast<const float*>(vals)[p]);
      if (colind[p] == r) c += alpha * a;
      else rad += fabs(alpha * a);
    }
    lo = fmin(lo, c - rad);
    hi = fmax(hi, c + rad);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&lo_hi[0], ordered_bits(lo));
    atomicMax(&lo_hi[1], ordered_bits(hi));
  }
}

} // namespace

extern "C" int trl_cuda_csr_gershgorin(trl_cuda_handle h, const trl_csr* A, double alpha, double beta, double* host_lo, double* host_hi)
{
  TRL_CHECK_HANDLE(h);
  if (!A || !host_lo || !host_hi) return set_error(h, TRL_EINVAL, "null pointer");
  *host_lo = *host_hi = beta;
  if (A->n == 0) return TRL_OK;
  unsigned long long* d = static_cast<unsigned long long*>(workspace(h, 64));
  if (!d) return TRL_ENOMEM;
  const unsigned long long init[2] = {~0ull, 0ull};
  if (int st = trl_cuda_memcpy(h, d, init, sizeof init, TRL_H2D)) return st;
  launch(k_gershgorin, grid_for(h, A->n, 256, 8), 256, 0, h->stream, A->n, A->rowptr, A->colind, A->values, A->value_dtype == TRL_F64, alpha, beta, d);
  if (int st = after_launch(h, "csr_gershgorin")) return st;
  unsigned long long bits[2] = {0, 0};
  if (int st = trl_cuda_memcpy(h, bits, d, sizeof bits, TRL_D2H)) return st;
  for (int i = 0; i < 2; ++i) {
    const unsigned long long u = (bits[i] >> 63) ? (bits[i] & 0x7fffffffffffffffull) : ~bits[i];
    std::memcpy(i == 0 ? host_lo : host_hi, &u, sizeof u);
  }
  return TRL_OK;
}

extern "C" int trl_cuda_csr_norm1(trl_cuda_handle h, const trl_csr* A, double alpha, double beta, double* host_out)
{
  TRL_CHECK_HANDLE(h);
  if (!A || !host_out) return set_error(h, TRL_EINVAL, "null pointer");
  *host_out = 0.0;
  if (A->n == 0) return TRL_OK;
  unsigned long long* d = static_cast<unsigned long long*>(workspace(h, 64));
  if (!d) return TRL_ENOMEM;
  cudaMemsetAsync(d, 0, sizeof(unsigned long long), h->stream);
  launch(k_norm1, grid_for(h, A->n, 256, 8), 256, 0, h->stream, A->n, A->rowptr, A->colind, A->values, A->value_dtype == TRL_F64, alpha, beta, d);
  if (int st = after_launch(h, "csr_norm1")) return st;
  unsigned long long bits = 0;
  if (int st = trl_cuda_memcpy(h, &bits, d, sizeof bits, TRL_D2H)) return st;
  std::memcpy(host_out, &bits, sizeof bits);
  return TRL_OK;
}
