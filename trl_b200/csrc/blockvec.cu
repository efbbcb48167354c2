// Block-vector kernels of the backend: elementwise ops, the multi-block inner product
// (block dot), the tall-skinny block GEMM behind mult / mult_transpose / mult_add /
// subtract_product / the CGS projection update / the thick-restart rotation, and
// Cholesky-QR. Contractions run on the FP64 tensor cores (DMMA m8n8k4); FP32 storage is
// widened to FP64 in registers, so products are exact and sums are FP64.
//
// Layout: a block vector is n x BS row-major; block j of a multivector at base + j*n*BS.
#include "common.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace {

constexpr int kThreads = 256; // 8 warps per CTA for every kernel in this file
constexpr int kWarps = kThreads / 32;

// ---------------------------------------------------------------- elementwise
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int width = 2;
};
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int width = 4;
};

template <typename T>
__device__ __forceinline__ void vsub(typename Vec16<T>::type& a, const typename Vec16<T>::type& b);
template <>
__device__ __forceinline__ void vsub<double>(double2& a, const double2& b)
{
  a.x -= b.x;
  a.y -= b.y;
}
template <>
__device__ __forceinline__ void vsub<float>(float4& a, const float4& b)
{
  a.x -= b.x;
  a.y -= b.y;
  a.z -= b.z;
  a.w -= b.w;
}

// X -= Y over `count` elements; vectorised when both pointers are 16-byte aligned.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_sub(T* __restrict__ X, const T* __restrict__ Y, int64_t count, int vec_ok)
{
  ::trl_detail::pdl_enter();
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::width;
  int64_t done = 0;
  if (vec_ok) {
    const int64_t nv = count / W;
    V* xv = reinterpret_cast<V*>(X);
    const V* yv = reinterpret_cast<const V*>(Y);
    for (int64_t i = tid; i < nv; i += stride) {
      V a = xv[i];
      vsub<T>(a, yv[i]);
      xv[i] = a;
    }
    done = nv * W;
  }
  for (int64_t i = done + tid; i < count; i += stride) X[i] -= Y[i];
}

template <typename D, typename S>
__global__ void __launch_bounds__(kThreads) k_convert(D* __restrict__ dst, const S* __restrict__ src, int64_t count)
{
  ::trl_detail::pdl_enter();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) dst[i] = static_cast<D>(src[i]);
}

// ---------------------------------------------------------------- block dot
// C_j = V_j^T W, j < nblk. Grid: x = chunk of JC blocks, y = chunk of rows.
// A warp takes G groups of 4 rows per iteration. All operand loads of the iteration are
// issued before the first DMMA (block indices beyond nblk are clamped to a valid block and
// their products discarded), so each warp keeps G*(JC+1)*NT 256-byte loads in flight.
// Per group: one DMMA m8n8k4 per (j, 8x8 output tile). Per-CTA sums go to
// partial[row_chunk][j][BS*BS]; k_reduce_partials adds the row chunks in a fixed order.
template <typename T, int BS, int JC, int G>
__global__ void __launch_bounds__(kThreads) k_block_dot(const T* __restrict__ V, int64_t vstride, int nblk, const T* __restrict__ W, int64_t n, int64_t rows_per_cta,
                                                        double* __restrict__ partial, const int* __restrict__ cond = nullptr)
{
  ::trl_detail::pdl_enter();
  if (cond && *cond == 0) return; // device-side skip (uniform over the grid)
  constexpr int NT = (BS + 7) / 8;
  constexpr int BB = BS * BS;
  __shared__ double red[kWarps][NT * NT * 64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int j0 = blockIdx.x * JC;
  const int64_t rb = static_cast<int64_t>(blockIdx.y) * rows_per_cta;
  const int64_t re = min(n, rb + rows_per_cta);

  double acc[JC][NT][NT][2];
#pragma unroll
  for (int jj = 0; jj < JC; ++jj)
#pragma unroll
    for (int a = 0; a < NT; ++a)
#pragma unroll
      for (int b = 0; b < NT; ++b) acc[jj][a][b][0] = acc[jj][a][b][1] = 0.0;

  const T* Vb[JC];
#pragma unroll
  for (int jj = 0; jj < JC; ++jj) Vb[jj] = V + static_cast<int64_t>(min(j0 + jj, nblk - 1)) * vstride;

  for (int64_t r0 = rb + warp * 4 * G; r0 < re; r0 += kWarps * 4 * G) {
    double bf[G][NT];
    double av[G][JC][NT];
#pragma unroll
    for (int q = 0; q < G; ++q) {
      const int64_t row = r0 + q * 4 + t4;
      const bool rok = row < re;
#pragma unroll
      for (int tk = 0; tk < NT; ++tk) {
        const int col = tk * 8 + g;
        bf[q][tk] = (rok && col < BS) ? ld_widen(W + row * BS + col) : 0.0;
      }
#pragma unroll
      for (int jj = 0; jj < JC; ++jj)
#pragma unroll
        for (int ti = 0; ti < NT; ++ti) {
          const int col = ti * 8 + g;
          av[q][jj][ti] = (rok && col < BS) ? ld_widen(Vb[jj] + row * BS + col) : 0.0;
        }
    }
#pragma unroll
    for (int q = 0; q < G; ++q)
#pragma unroll
      for (int jj = 0; jj < JC; ++jj) {
        if (j0 + jj < nblk) {
#pragma unroll
          for (int ti = 0; ti < NT; ++ti)
#pragma unroll
            for (int tk = 0; tk < NT; ++tk) dmma_m8n8k4(acc[jj][ti][tk][0], acc[jj][ti][tk][1], av[q][jj][ti], bf[q][tk]);
        }
      }
  }

  // cross-warp reduction, one block j at a time
#pragma unroll
  for (int jj = 0; jj < JC; ++jj) {
    if (j0 + jj >= nblk) break;
#pragma unroll
    for (int ti = 0; ti < NT; ++ti)
#pragma unroll
      for (int tk = 0; tk < NT; ++tk) {
        red[warp][(ti * NT + tk) * 64 + g * 8 + 2 * t4 + 0] = acc[jj][ti][tk][0];
        red[warp][(ti * NT + tk) * 64 + g * 8 + 2 * t4 + 1] = acc[jj][ti][tk][1];
      }
    __syncthreads();
    for (int e = threadIdx.x; e < NT * NT * 64; e += kThreads) {
      const int tile = e >> 6, within = e & 63;
      const int row = (tile / NT) * 8 + (within >> 3);
      const int col = (tile % NT) * 8 + (within & 7);
      if (row < BS && col < BS) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += red[w][e];
        partial[(static_cast<int64_t>(blockIdx.y) * nblk + j0 + jj) * BB + row * BS + col] = s;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- block dot, bulk-copy pipeline
// Same result as k_block_dot, for BS*sizeof(T) a multiple of 16 bytes. The CTA walks its
// row range in tiles of R rows (4 KB per block tile). Thread 0 streams the W tile and the
// tiles of the JC blocks of V into an S-stage shared-memory ring with 1-D bulk copies that
// complete on a per-stage "full" mbarrier; the 8 warps read DMMA fragments from shared
// memory and release the stage on its "empty" mbarrier. HBM traffic is a continuous stream
// of 4 KB copies, independent of register pressure and of the element width.
// Waits are bounded (mbar_wait): on a timeout the status word records TRL_DEV_TIMEOUT, the
// threads leave the tile loop, and thread 0 waits (bounded) for the copies it issued.
template <typename T, int BS, int TB>
struct BulkTile {
  static constexpr int R = TB / (BS * static_cast<int>(sizeof(T))); // rows per tile (TB bytes per block tile)
  static constexpr int ELEMS = R * BS;
};

template <typename T, int BS, int JC, int S, int TB>
__global__ void __launch_bounds__(kThreads) k_block_dot_bulk(const T* __restrict__ V, int64_t vstride, int nblk, const T* __restrict__ W, int64_t n, int64_t rows_per_cta,
                                                             double* __restrict__ partial, int* status, const int* __restrict__ cond)
{
  ::trl_detail::pdl_enter();
  if (cond && *cond == 0) return; // device-side skip (uniform over the grid)
  constexpr int NT = (BS + 7) / 8;
  constexpr int BB = BS * BS;
  constexpr int R = BulkTile<T, BS, TB>::R;
  constexpr int TILE = BulkTile<T, BS, TB>::ELEMS;
  constexpr int GPW = R / (kWarps * 4); // 4-row groups per warp per tile
  static_assert(GPW >= 1 && R % (kWarps * 4) == 0, "tile rows must cover the CTA's warps");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* tiles = reinterpret_cast<T*>(smem_raw); // [S][JC + 1][TILE]: slot 0 is W
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(S) * (JC + 1) * TILE * sizeof(T));
  uint64_t* empty = full + S;
  __shared__ double red[kWarps][NT * NT * 64];

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int j0 = blockIdx.x * JC;
  const int jn = min(JC, nblk - j0);
  const int64_t rb = static_cast<int64_t>(blockIdx.y) * rows_per_cta;
  const int64_t re = min(n, rb + rows_per_cta);
  const int ntiles = re > rb ? static_cast<int>((re - rb + R - 1) / R) : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kWarps);
    }
    mbar_init_fence();
  }
  __syncthreads();

  int issued = 0; // thread 0: tiles whose copies were started
  auto issue = [&](int t) {
    const int s = t % S;
    const int64_t r0 = rb + static_cast<int64_t>(t) * R;
    const uint32_t bytes = static_cast<uint32_t>(min(static_cast<int64_t>(R), re - r0) * BS * sizeof(T));
    T* st = tiles + static_cast<size_t>(s) * (JC + 1) * TILE;
    mbar_arrive_expect_tx(&full[s], bytes * static_cast<uint32_t>(jn + 1));
    bulk_g2s(st, W + r0 * BS, bytes, &full[s]);
    for (int jj = 0; jj < jn; ++jj) bulk_g2s(st + (jj + 1) * TILE, V + static_cast<int64_t>(j0 + jj) * vstride + r0 * BS, bytes, &full[s]);
    issued = t + 1;
  };
  if (threadIdx.x == 0)
    for (int t = 0; t < min(S - 1, ntiles); ++t) issue(t);

  double acc[JC][NT][NT][2];
#pragma unroll
  for (int jj = 0; jj < JC; ++jj)
#pragma unroll
    for (int a = 0; a < NT; ++a)
#pragma unroll
      for (int b = 0; b < NT; ++b) acc[jj][a][b][0] = acc[jj][a][b][1] = 0.0;

  int consumed = 0;
  for (int t = 0; t < ntiles; ++t) {
    if (threadIdx.x == 0 && t + S - 1 < ntiles) {
      const int tn = t + S - 1; // refill the slot that tile t-1 used
      if (tn < S || mbar_wait(&empty[tn % S], static_cast<uint32_t>((tn - S) / S) & 1u, status)) issue(tn);
    }
    const int s = t % S;
    if (!mbar_wait(&full[s], static_cast<uint32_t>(t / S) & 1u, status)) break;
    const T* st = tiles + static_cast<size_t>(s) * (JC + 1) * TILE;
    const int rows = static_cast<int>(min(static_cast<int64_t>(R), re - (rb + static_cast<int64_t>(t) * R)));
#pragma unroll
    for (int q = 0; q < GPW; ++q) {
      const int lr = (warp * GPW + q) * 4 + t4;
      const bool rok = lr < rows;
      double bf[NT];
#pragma unroll
      for (int tk = 0; tk < NT; ++tk) {
        const int col = tk * 8 + g;
        bf[tk] = (rok && col < BS) ? static_cast<double>(st[lr * BS + col]) : 0.0;
      }
#pragma unroll
      for (int jj = 0; jj < JC; ++jj) {
        if (jj < jn) {
#pragma unroll
          for (int ti = 0; ti < NT; ++ti) {
            const int col = ti * 8 + g;
            const double a = (rok && col < BS) ? static_cast<double>(st[(jj + 1) * TILE + lr * BS + col]) : 0.0;
#pragma unroll
            for (int tk = 0; tk < NT; ++tk) dmma_m8n8k4(acc[jj][ti][tk][0], acc[jj][ti][tk][1], a, bf[tk]);
          }
        }
      }
    }
    __syncwarp(); // the DMMAs above consumed every lane's shared-memory reads
    if (lane == 0) mbar_arrive(&empty[s]);
    consumed = t + 1;
  }
  if (threadIdx.x == 0) // after an aborted loop: let the copies already started land
    for (int t = consumed; t < issued; ++t) mbar_wait(&full[t % S], static_cast<uint32_t>(t / S) & 1u, status, 1u << 20);

#pragma unroll
  for (int jj = 0; jj < JC; ++jj) {
    if (jj >= jn) break;
#pragma unroll
    for (int ti = 0; ti < NT; ++ti)
#pragma unroll
      for (int tk = 0; tk < NT; ++tk) {
        red[warp][(ti * NT + tk) * 64 + g * 8 + 2 * t4 + 0] = acc[jj][ti][tk][0];
        red[warp][(ti * NT + tk) * 64 + g * 8 + 2 * t4 + 1] = acc[jj][ti][tk][1];
      }
    __syncthreads();
    for (int e = threadIdx.x; e < NT * NT * 64; e += kThreads) {
      const int tile = e >> 6, within = e & 63;
      const int row = (tile / NT) * 8 + (within >> 3);
      const int col = (tile % NT) * 8 + (within & 7);
      if (row < BS && col < BS) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum += red[w][e];
        partial[(static_cast<int64_t>(blockIdx.y) * nblk + j0 + jj) * BB + row * BS + col] = sum;
      }
    }
    __syncthreads();
  }
}

// Sum of partial[c][e] over the chunks c = s, s + SL, s + 2 SL, ... of one slice. Eight
// loads are issued before the adds that consume them (a thread issues in order, so each
// batch is one dependent memory round: ~600 partials take 3 rounds, not 5); eight
// accumulators, combined in a fixed tree, so the result does not depend on scheduling.
template <int SL>
__device__ __forceinline__ double slice_sum(const double* __restrict__ partial, int chunks, int64_t len, int64_t e, int s)
{
  constexpr int U = 8;
  double a[U];
#pragma unroll
  for (int u = 0; u < U; ++u) a[u] = 0.0;
  for (int c = s; c < chunks; c += U * SL) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int cu = c + u * SL;
      v[u] = cu < chunks ? partial[static_cast<int64_t>(cu) * len + e] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) a[u] += v[u];
  }
  return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}

// out[e] = sum_c partial[c][e]: OPC outputs per CTA, SL = 1024 / OPC slices of the chunk
// range per output (slice_sum); the slices are combined in a fixed order, so the result
// does not depend on scheduling. OPC = 32 for long outputs (one warp per slice, coalesced);
// OPC = 8 for short ones (the b x b blocks of one or a few basis blocks): eight times the
// CTAs and a quarter of the loads per thread, so that ~600 partials take one memory round.
constexpr int kRedThreads = 1024;
template <int OPC>
__global__ void __launch_bounds__(kRedThreads) k_reduce_partials(const double* __restrict__ partial, int chunks, int64_t len, double* __restrict__ out,
                                                                 const int* __restrict__ cond)
{
  ::trl_detail::pdl_enter();
  if (cond && *cond == 0) return;
  constexpr int SL = kRedThreads / OPC;
  __shared__ double part[SL][OPC + 1];
  const int o = threadIdx.x % OPC, s = threadIdx.x / OPC;
  const int64_t e = static_cast<int64_t>(blockIdx.x) * OPC + o;
  part[s][o] = e < len ? slice_sum<SL>(partial, chunks, len, e, s) : 0.0;
  __syncthreads();
  if (s == 0 && e < len) {
    double t = 0.0;
#pragma unroll 8
    for (int q = 0; q < SL; ++q) t += part[q][o];
    out[e] = t;
  }
}

// Launches the fixed-order reduction of `chunks` partial rows of `len` doubles into out.
inline cudaError_t launch_reduce(cudaStream_t stream, const double* partial, int64_t chunks, int64_t len, double* out, const int* cond)
{
  if (len <= 1024 && chunks > 128)
    return ::trl_detail::launch(k_reduce_partials<8>, static_cast<unsigned>((len + 7) / 8), kRedThreads, 0, stream, partial, static_cast<int>(chunks), len, out, cond);
  return ::trl_detail::launch(k_reduce_partials<32>, static_cast<unsigned>((len + 31) / 32), kRedThreads, 0, stream, partial, static_cast<int>(chunks), len, out, cond);
}

// ---------------------------------------------------------------- block GEMM
// out_j = (accumulate ? out_j : 0) + sign * sum_{i<MB} in_i * Coef(i, j)   for j < NB <= NBMAX
// Coef(i, j) = coef + (i*ldc + j)*BS*BS (row-major BS x BS, or its transpose).
// A warp owns RT 8-row tiles at a time and walks the input blocks U at a time: the
// A-fragment loads of U blocks x RT tiles (from `in`, HBM) are all issued before the DMMAs
// that consume them (indices past MB are clamped and their products skipped). B fragments
// come from the tiny coefficient array (L1-resident) and are shared by the RT tiles.
// `in` and `out` may alias when MB = NB = 1 (in-place X <- X U^{-1}): a warp reads all its
// rows before it writes them, and no other warp touches those rows.
template <typename T, int BS, int NBMAX, int RT, int U>
__global__ void __launch_bounds__(kThreads) k_block_gemm(const T* in, int64_t istride, int MB, const double* __restrict__ coef, int ldc, int transpose_coef, T* out,
                                                         int64_t ostride, int NB, int64_t n, int accumulate, double sign)
{
  ::trl_detail::pdl_enter();
  constexpr int NT = (BS + 7) / 8;
  constexpr int KS = (BS + 3) / 4;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int64_t warp_global = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  const int64_t warp_stride = static_cast<int64_t>(gridDim.x) * kWarps;

  for (int64_t r0 = warp_global * 8 * RT; r0 < n; r0 += warp_stride * 8 * RT) {
    double acc[RT][NBMAX][NT][2];
#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const int64_t row = r0 + r * 8 + g;
      const bool rok = row < n;
#pragma unroll
      for (int jb = 0; jb < NBMAX; ++jb)
#pragma unroll
        for (int t = 0; t < NT; ++t)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int col = t * 8 + 2 * t4 + i;
            acc[r][jb][t][i] = (accumulate && jb < NB && rok && col < BS) ? static_cast<double>(out[jb * ostride + row * BS + col]) : 0.0;
          }
    }

    for (int ib0 = 0; ib0 < MB; ib0 += U) {
      double a[U][RT][KS];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const T* A = in + static_cast<int64_t>(min(ib0 + u, MB - 1)) * istride;
#pragma unroll
        for (int r = 0; r < RT; ++r) {
          const int64_t row = r0 + r * 8 + g;
#pragma unroll
          for (int ks = 0; ks < KS; ++ks) {
            const int kcol = ks * 4 + t4;
            a[u][r][ks] = (row < n && kcol < BS) ? static_cast<double>(A[row * BS + kcol]) : 0.0;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (ib0 + u < MB) {
          const double* Crow = coef + static_cast<int64_t>(ib0 + u) * ldc * (BS * BS);
#pragma unroll
          for (int ks = 0; ks < KS; ++ks)
#pragma unroll
            for (int jb = 0; jb < NBMAX; ++jb) {
              if (jb < NB) {
                const double* Cb = Crow + jb * (BS * BS);
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                  const int krow = ks * 4 + t4, ncol = t * 8 + g;
                  double b = 0.0;
                  if (krow < BS && ncol < BS) b = sign * __ldg(transpose_coef ? Cb + ncol * BS + krow : Cb + krow * BS + ncol);
#pragma unroll
                  for (int r = 0; r < RT; ++r) dmma_m8n8k4(acc[r][jb][t][0], acc[r][jb][t][1], a[u][r][ks], b);
                }
              }
            }
        }
      }
    }

#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const int64_t row = r0 + r * 8 + g;
#pragma unroll
      for (int jb = 0; jb < NBMAX; ++jb)
#pragma unroll
        for (int t = 0; t < NT; ++t)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int col = t * 8 + 2 * t4 + i;
            if (jb < NB && row < n && col < BS) out[jb * ostride + row * BS + col] = static_cast<T>(acc[r][jb][t][i]);
          }
    }
  }
}

// ---------------------------------------------------------------- restart rotation
// W_j = sum_{i<m} V_i Y(i,j) for the output columns [c0, c0 + 8*NTC) of the N = k*BS columns
// (one chunk of output columns per launch). As a GEMM, out[rows x N] = V[rows x K] * Yhat[K x N]
// with K = m*BS: 2*n*K*N flops over (K + N)*n elements, ~9 flop/B at the thick restart's
// shapes, so the kernel is bound by the FP64 DMMA rate rather than by HBM.
// The chunk of Yhat lives in shared memory in DMMA B-fragment order (for every k-step of 4
// rows and n-tile of 8 columns the 32 values in lane order: one conflict-free 256-byte load
// per fragment) and is loaded once per CTA. Each warp owns RT tiles of 8 rows and streams the
// m input blocks through a register ring D blocks deep, so every load is issued D blocks
// before the DMMAs that consume it.
constexpr int kRotThreads = 512;

template <typename T, int BS, int NTC, int RT, int D>
__global__ void __launch_bounds__(kRotThreads, 1) k_rotate(const T* __restrict__ V, int64_t vstride, int m, const double* __restrict__ Y, int ldy, int N, int c0,
                                                           T* __restrict__ W, int64_t wstride, int64_t n)
{
  ::trl_detail::pdl_enter();
  constexpr int KSB = BS / 4; // k-steps per input block
  extern __shared__ double sY[];
  const int ks_total = m * KSB;
  for (int idx = threadIdx.x; idx < ks_total * NTC * 32; idx += blockDim.x) {
    const int ln = idx & 31, f = idx >> 5;
    const int nt = f % NTC, ks = f / NTC;
    const int krow = ks * 4 + (ln & 3), col = c0 + nt * 8 + (ln >> 2);
    double v = 0.0;
    if (col < N) {
      const int i = krow / BS, r = krow % BS, j = col / BS, cc = col % BS;
      v = Y[(static_cast<int64_t>(i) * ldy + j) * (BS * BS) + r * BS + cc];
    }
    sY[idx] = v;
  }
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int64_t warp = static_cast<int64_t>(blockIdx.x) * (kRotThreads / 32) + (threadIdx.x >> 5);
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (kRotThreads / 32);

  for (int64_t r0 = warp * 8 * RT; r0 < n; r0 += nwarps * 8 * RT) {
    double acc[RT][NTC][2];
#pragma unroll
    for (int rt = 0; rt < RT; ++rt)
#pragma unroll
      for (int nt = 0; nt < NTC; ++nt) acc[rt][nt][0] = acc[rt][nt][1] = 0.0;

    double a[D][RT][KSB];
    auto load = [&](double(&dst)[RT][KSB], int blk) {
#pragma unroll
      for (int rt = 0; rt < RT; ++rt) {
        const int64_t row = r0 + rt * 8 + g;
#pragma unroll
        for (int ks = 0; ks < KSB; ++ks)
          dst[rt][ks] = (blk < m && row < n) ? static_cast<double>(V[static_cast<int64_t>(blk) * vstride + row * BS + ks * 4 + t4]) : 0.0;
      }
    };
#pragma unroll
    for (int d = 0; d < D; ++d) load(a[d], d);

    for (int ib = 0; ib < m; ib += D) {
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const int i = ib + d;
        if (i < m) {
#pragma unroll
          for (int ks = 0; ks < KSB; ++ks) {
            const double* bf = sY + static_cast<size_t>((i * KSB + ks) * NTC) * 32 + lane;
#pragma unroll
            for (int nt = 0; nt < NTC; ++nt) {
              const double b = bf[nt * 32];
#pragma unroll
              for (int rt = 0; rt < RT; ++rt) dmma_m8n8k4(acc[rt][nt][0], acc[rt][nt][1], a[d][rt][ks], b);
            }
          }
        }
        load(a[d], i + D);
      }
    }

#pragma unroll
    for (int rt = 0; rt < RT; ++rt) {
      const int64_t row = r0 + rt * 8 + g;
      if (row >= n) continue;
#pragma unroll
      for (int nt = 0; nt < NTC; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = c0 + nt * 8 + 2 * t4 + e;
          if (col < N) W[static_cast<int64_t>(col / BS) * wstride + row * BS + (col % BS)] = static_cast<T>(acc[rt][nt][e]);
        }
    }
  }
}

// KS adjacent elements p[0..KS) (p aligned to KS * sizeof(T) when that is 8 or 16 bytes),
// in as few loads as possible; columns past BS are never requested.
template <typename T, int KS>
__device__ __forceinline__ void load_cols(const T* p, T (&v)[KS])
{
  if constexpr (sizeof(T) == 8 && KS == 2) {
    const double2 q = *reinterpret_cast<const double2*>(p);
    v[0] = q.x;
    v[1] = q.y;
  }
  else if constexpr (sizeof(T) == 8 && KS == 4) {
    const double2 q0 = *reinterpret_cast<const double2*>(p), q1 = *reinterpret_cast<const double2*>(p + 2);
    v[0] = q0.x;
    v[1] = q0.y;
    v[2] = q1.x;
    v[3] = q1.y;
  }
  else if constexpr (sizeof(T) == 4 && KS == 2) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    v[0] = q.x;
    v[1] = q.y;
  }
  else if constexpr (sizeof(T) == 4 && KS == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
  }
  else {
#pragma unroll
    for (int i = 0; i < KS; ++i) v[i] = p[i];
  }
}

// ---------------------------------------------------------------- update + Gram in one pass
// out = (accumulate ? out : 0) + sign * sum_{i<MB} in_i Coef(i),  Coef(i) = coef + i*BS*BS,
// and in the same pass the Gram matrix out^T out of the values as stored (rounded to T):
// each warp stages its finished rows in shared memory, re-reads them in DMMA fragment
// layout (k = rows) and accumulates the BS x BS Gram; per-CTA sums go to
// gram_partial[blockIdx.x][BS*BS]. When cond is given and *cond == 0 the kernel does
// nothing (a device-side decision: no host round trip). `in` and `out` may alias for MB = 1.
template <typename T, int BS, int RT, int U>
__global__ void __launch_bounds__(kThreads) k_update_gram(const T* in, int64_t istride, int MB, const double* __restrict__ coef, T* out, int64_t n, int accumulate, double sign,
                                                          double* __restrict__ gram_partial, const int* __restrict__ cond)
{
  ::trl_detail::pdl_enter();
  if (cond && *cond == 0) return;
  constexpr int NT = (BS + 7) / 8;
  constexpr int KS = (BS + 3) / 4;
  __shared__ double stage[kWarps][RT * 8 * BS];
  __shared__ double red[kWarps][NT * NT * 64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int64_t warp_global = static_cast<int64_t>(blockIdx.x) * kWarps + warp;
  const int64_t warp_stride = static_cast<int64_t>(gridDim.x) * kWarps;
  double gacc[NT][NT][2];
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b) gacc[a][b][0] = gacc[a][b][1] = 0.0;

  for (int64_t r0 = warp_global * 8 * RT; r0 < n; r0 += warp_stride * 8 * RT) {
    double acc[RT][NT][2];
#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const int64_t row = r0 + r * 8 + g;
#pragma unroll
      for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int col = t * 8 + 2 * t4 + i;
          acc[r][t][i] = (accumulate && row < n && col < BS) ? static_cast<double>(out[row * BS + col]) : 0.0;
        }
    }
    for (int ib0 = 0; ib0 < MB; ib0 += U) {
      // k is permuted so that lane t4 owns the KS adjacent columns t4*KS .. t4*KS+KS-1 of
      // its row (one vector load); the values stay in the storage type until the DMMA
      T a[U][RT][KS];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const T* A = in + static_cast<int64_t>(min(ib0 + u, MB - 1)) * istride;
#pragma unroll
        for (int r = 0; r < RT; ++r) {
          const int64_t row = r0 + r * 8 + g;
          if (row < n && t4 * KS < BS) load_cols<T, KS>(A + row * BS + t4 * KS, a[u][r]);
          else
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) a[u][r][ks] = T(0);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (ib0 + u < MB) {
          const double* Cb = coef + static_cast<int64_t>(ib0 + u) * (BS * BS);
#pragma unroll
          for (int ks = 0; ks < KS; ++ks)
#pragma unroll
            for (int t = 0; t < NT; ++t) {
              const int krow = t4 * KS + ks, ncol = t * 8 + g;
              const double b = (krow < BS && ncol < BS) ? sign * __ldg(Cb + krow * BS + ncol) : 0.0;
#pragma unroll
              for (int r = 0; r < RT; ++r) dmma_m8n8k4(acc[r][t][0], acc[r][t][1], static_cast<double>(a[u][r][ks]), b);
            }
        }
      }
    }
    // store, and stage the stored values for the Gram
#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const int64_t row = r0 + r * 8 + g;
#pragma unroll
      for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int col = t * 8 + 2 * t4 + i;
          if (col < BS) {
            const T v = static_cast<T>(acc[r][t][i]);
            if (row < n) out[row * BS + col] = v;
            stage[warp][(r * 8 + g) * BS + col] = row < n ? static_cast<double>(v) : 0.0;
          }
        }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2 * RT; ++q) { // groups of 4 staged rows = the DMMA k dimension
      const int lr = q * 4 + t4;
      double bf[NT];
#pragma unroll
      for (int tk = 0; tk < NT; ++tk) bf[tk] = (tk * 8 + g < BS) ? stage[warp][lr * BS + tk * 8 + g] : 0.0;
#pragma unroll
      for (int ti = 0; ti < NT; ++ti) {
        const double av = (ti * 8 + g < BS) ? stage[warp][lr * BS + ti * 8 + g] : 0.0;
#pragma unroll
        for (int tk = 0; tk < NT; ++tk) dmma_m8n8k4(gacc[ti][tk][0], gacc[ti][tk][1], av, bf[tk]);
      }
    }
    __syncwarp();
  }
  // cross-warp reduction of the Gram
#pragma unroll
  for (int ti = 0; ti < NT; ++ti)
#pragma unroll
    for (int tk = 0; tk < NT; ++tk) {
      red[warp][(ti * NT + tk) * 64 + g * 8 + 2 * t4 + 0] = gacc[ti][tk][0];
      red[warp][(ti * NT + tk) * 64 + g * 8 + 2 * t4 + 1] = gacc[ti][tk][1];
    }
  __syncthreads();
  for (int e = threadIdx.x; e < NT * NT * 64; e += kThreads) {
    const int tile = e >> 6, within = e & 63;
    const int row = (tile / NT) * 8 + (within >> 3);
    const int col = (tile % NT) * 8 + (within & 7);
    if (row < BS && col < BS) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) s += red[w][e];
      gram_partial[static_cast<int64_t>(blockIdx.x) * BS * BS + row * BS + col] = s;
    }
  }
}

// DGKS criterion (Daniel, Gragg, Kaufman & Stewart 1976): a second Gram-Schmidt pass is
// needed when some column kept less than eta of its norm through the first pass.
template <int BS>
__global__ void k_dgks_flag(const double* __restrict__ G_before, const double* __restrict__ G_after, double eta2, int* __restrict__ flag)
{
  ::trl_detail::pdl_enter();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int f = 0;
  for (int c = 0; c < BS; ++c) f |= (G_after[c * BS + c] < eta2 * G_before[c * BS + c]);
  *flag = f;
}

// flag = ||E||_F^2 > thr2 * trace(G): the sketch S^T W (E) says W's components along the
// basis exceed thr relative to W's norm (G = W^T W). With `pair` (a word kept across calls),
// a step whose test fired also projects the next one: pair = this step's test.
template <int BS>
__global__ void k_sketch_flag(const double* __restrict__ E, const double* __restrict__ G, double thr2, int* __restrict__ flag, int* __restrict__ pair)
{
  ::trl_detail::pdl_enter();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double e2 = 0.0, tr = 0.0;
  for (int i = 0; i < BS * BS; ++i) e2 = fma(E[i], E[i], e2);
  for (int c = 0; c < BS; ++c) tr += G[c * BS + c];
  const int fired = !(e2 <= thr2 * tr); // NaN counts as loss
  int f = fired;
  if (pair) {
    f |= (*pair != 0) ? 2 : 0; // bit 1: forced by the previous step
    *pair = fired;
  }
  *flag = f;
}

// flag2 = flag1 && (a column kept less than eta of its norm through pass 1)
template <int BS>
__global__ void k_dgks_flag_after(const int* __restrict__ flag1, const double* __restrict__ G_before, const double* __restrict__ G_after, double eta2, int* __restrict__ flag2)
{
  ::trl_detail::pdl_enter();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int f = 0;
  if (*flag1)
    for (int c = 0; c < BS; ++c) f |= (G_after[c * BS + c] < eta2 * G_before[c * BS + c]);
  *flag2 = f;
}

// dst = *f2 ? c : (*f1 ? b : a)  (BS x BS)
__global__ void k_select_block3(const int* __restrict__ f1, const int* __restrict__ f2, const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
                                double* __restrict__ dst, int count)
{
  ::trl_detail::pdl_enter();
  const int e = threadIdx.x;
  if (e < count) dst[e] = *f2 ? c[e] : (*f1 ? b[e] : a[e]);
}

// dst = *flag ? a : b  (BS x BS)
__global__ void k_select_block(const int* __restrict__ flag, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ dst, int count)
{
  ::trl_detail::pdl_enter();
  const int e = threadIdx.x;
  if (e < count) dst[e] = *flag ? a[e] : b[e];
}

// ---------------------------------------------------------------- small Cholesky
// Gram matrix G from `chunks` partial sums (chunks = 0: G given), then G = L L^T reading
// the lower triangle, Uinv = L^{-T} for the apply, and R <- L^T (first pass) or
// R <- L^T R (so that X_in = X_out R across passes). All in shared memory; the factor and
// the inverse are column-parallel over one warp. A pivot <= 0 (or NaN) records
// TRL_DEV_CHOLESKY and writes Uinv = I, leaving the apply a no-op.
// With partial sums the reduction is spread over ceil(BS^2 / kFactorOPC) CTAs, each
// summing kFactorOPC entries of G in a fixed order into gsum; the CTA that finishes last
// (a ticket counter, left at zero again) factors. Every entry is summed by one CTA in one
// order, so the result does not depend on scheduling.
constexpr int kFactorOPC = 8;
template <int BS>
__global__ void __launch_bounds__(kRedThreads) k_gram_factor(const double* __restrict__ src, int chunks, double* __restrict__ Uinv, double* __restrict__ R, int first,
                                                             int* status, double* gsum, unsigned* ticket)
{
  ::trl_detail::pdl_enter();
  constexpr int OPC = kFactorOPC;
  constexpr int SL = kRedThreads / OPC; // slices of the chunk range per entry
  __shared__ double G[BS * BS], L[BS][BS + 1], Li[BS][BS + 1], Ro[BS * BS];
  __shared__ double part[SL][OPC + 1];
  __shared__ int bad, last;
  const int tid = threadIdx.x;
  // 1. G (the same fixed-order reduction as k_reduce_partials<8>)
  if (chunks > 0) {
    const int o = tid % OPC, s = tid / OPC, e = static_cast<int>(blockIdx.x) * OPC + o;
    part[s][o] = e < BS * BS ? slice_sum<SL>(src, chunks, BS * BS, e, s) : 0.0;
    __syncthreads();
    if (s == 0 && e < BS * BS) {
      double t = 0.0;
#pragma unroll 8
      for (int q = 0; q < SL; ++q) t += part[q][o];
      gsum[e] = t;
    }
    if (gridDim.x > 1) {
      __threadfence(); // this CTA's entries of gsum are visible before its ticket is taken
      __syncthreads();
      if (tid == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
      __syncthreads();
      if (!last) return;
      __threadfence();
      if (tid == 0) *ticket = 0u;
    }
    else
      __syncthreads();
    for (int e = tid; e < BS * BS; e += blockDim.x) G[e] = __ldcg(gsum + e); // L2: written by other CTAs
  }
  else {
    for (int e = tid; e < BS * BS; e += blockDim.x) G[e] = src[e];
  }
  for (int e = tid; e < BS * BS; e += blockDim.x) Ro[e] = R[e];
  if (tid == 0) bad = 0;
  __syncthreads();
  if (tid < 32) {
    const int lane = tid;
    // 2. L: column by column; lane i < BS owns row i
    for (int j = 0; j < BS; ++j) {
      if (lane == j) {
        double d = G[j * BS + j];
        for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
        if (!(d > 0.0)) bad = 1;
        L[j][j] = d > 0.0 ? sqrt(d) : 1.0;
      }
      __syncwarp();
      if (lane > j && lane < BS) {
        double s = G[lane * BS + j];
        for (int k = 0; k < j; ++k) s -= L[lane][k] * L[j][k];
        L[lane][j] = s / L[j][j];
      }
      if (lane < j) L[lane][j] = 0.0;
      __syncwarp();
    }
    // 3. Li = L^{-1} (lower): lane c owns column c, forward substitution
    if (lane < BS) {
      const int c = lane;
      for (int i = 0; i < BS; ++i) {
        if (i < c) {
          Li[i][c] = 0.0;
          continue;
        }
        double s = (i == c) ? 1.0 : 0.0;
        for (int k = c; k < i; ++k) s -= L[i][k] * Li[k][c];
        Li[i][c] = s / L[i][i];
      }
    }
    __syncwarp();
    // 4. outputs: Uinv = Li^T; R (lane i owns row i)
    if (lane < BS) {
      const int i = lane;
      for (int c = 0; c < BS; ++c) Uinv[i * BS + c] = bad ? (i == c ? 1.0 : 0.0) : Li[c][i];
      if (!bad) {
        for (int c = 0; c < BS; ++c) {
          double s;
          if (first) {
            s = (c >= i) ? L[c][i] : 0.0;
          }
          else {
            s = 0.0;
            for (int k = i; k <= c; ++k) s += L[k][i] * Ro[k * BS + c];
            if (c < i) s = 0.0;
          }
          R[i * BS + c] = s;
        }
      }
    }
    if (lane == 0 && bad) atomicOr(status, TRL_DEV_CHOLESKY);
  }
}


} // namespace

using namespace trl_detail;

// ---------------------------------------------------------------- launchers
namespace trl_detail {

template <typename T, int BS, int JC, int G>
int launch_block_dot_jc(trl_cuda_context* h, const T* V, int nblk, const T* W, int64_t n, double* C, const int* cond)
{
  const int64_t len = static_cast<int64_t>(nblk) * BS * BS;
  const int gj = (nblk + JC - 1) / JC;
  // about 4 CTAs per SM in total, 512+ rows per CTA
  int64_t target = static_cast<int64_t>(h->num_sms) * 4 / gj;
  if (target < 1) target = 1;
  int64_t max_chunks = (n + 511) / 512;
  int64_t chunks = target < max_chunks ? target : max_chunks;
  if (chunks < 1) chunks = 1;
  int64_t rows_per_cta = (n + chunks - 1) / chunks;
  constexpr int step = kWarps * 4 * G; // rows one CTA iteration covers
  rows_per_cta = (rows_per_cta + step - 1) / step * step;
  chunks = (n + rows_per_cta - 1) / rows_per_cta;
  double* partial = static_cast<double*>(workspace(h, static_cast<size_t>(chunks) * len * sizeof(double)));
  if (!partial) return TRL_ENOMEM;
  dim3 grid(gj, static_cast<unsigned>(chunks));
  launch(k_block_dot<T, BS, JC, G>, grid, kThreads, 0, h->stream, V, n * BS, nblk, W, n, rows_per_cta, partial, cond);
  int st = after_launch(h, "block_dot");
  if (st) return st;
  launch_reduce(h->stream, partial, chunks, len, C, cond);
  return after_launch(h, "block_dot reduce");
}

// C = [A, B]^T W (2 blocks of bs x bs) for two blocks anywhere in memory, reading W once:
// the register kernel's blocks are V and V + vstride.
template <typename T, int BS>
int launch_block_dot_two(trl_cuda_context* h, const T* A, const T* B, const T* W, int64_t n, double* C)
{
  constexpr int JC = 2, G = 4;
  constexpr int64_t len = 2 * BS * BS;
  int64_t target = static_cast<int64_t>(h->num_sms) * 4;
  int64_t max_chunks = (n + 511) / 512;
  int64_t chunks = target < max_chunks ? target : max_chunks;
  if (chunks < 1) chunks = 1;
  int64_t rows_per_cta = (n + chunks - 1) / chunks;
  constexpr int step = kWarps * 4 * G;
  rows_per_cta = (rows_per_cta + step - 1) / step * step;
  chunks = (n + rows_per_cta - 1) / rows_per_cta;
  double* partial = static_cast<double*>(workspace(h, static_cast<size_t>(chunks) * len * sizeof(double)));
  if (!partial) return TRL_ENOMEM;
  const int64_t vstride = B - A; // elements between the two blocks
  launch(k_block_dot<T, BS, JC, G>, dim3(1, static_cast<unsigned>(chunks)), kThreads, 0, h->stream, A, vstride, 2, W, n, rows_per_cta, partial, nullptr);
  int st = after_launch(h, "block_dot");
  if (st) return st;
  launch_reduce(h->stream, partial, chunks, len, C, nullptr);
  return after_launch(h, "block_dot reduce");
}

template <typename T, int BS, int JC, int S, int TB>
int launch_block_dot_bulk(trl_cuda_context* h, const T* V, int nblk, const T* W, int64_t n, double* C, const int* cond)
{
  constexpr int R = BulkTile<T, BS, TB>::R;
  constexpr size_t smem = static_cast<size_t>(S) * (JC + 1) * BulkTile<T, BS, TB>::ELEMS * sizeof(T) + 2 * S * sizeof(uint64_t);
  // the shared-memory attribute belongs to the current device: set it on every call
  if (cudaFuncSetAttribute(k_block_dot_bulk<T, BS, JC, S, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(h, TRL_ECUDA, "block dot: %zu bytes of shared memory refused", smem);
  }
  static int resident = 0; // CTAs per SM at this shared-memory size (queried once; same on every B200)
  if (resident == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_block_dot_bulk<T, BS, JC, S, TB>, kThreads, smem) != cudaSuccess || resident < 1) resident = 1;
    cudaGetLastError();
  }
  const int64_t len = static_cast<int64_t>(nblk) * BS * BS;
  const int gj = (nblk + JC - 1) / JC;
  int64_t chunks = static_cast<int64_t>(h->num_sms) * resident / gj;
  if (chunks < 1) chunks = 1;
  const int64_t max_chunks = (n + 2 * R - 1) / (2 * R); // at least two tiles per CTA
  if (chunks > max_chunks) chunks = max_chunks;
  int64_t rows_per_cta = (n + chunks - 1) / chunks;
  rows_per_cta = (rows_per_cta + R - 1) / R * R;
  chunks = (n + rows_per_cta - 1) / rows_per_cta;
  double* partial = static_cast<double*>(workspace(h, static_cast<size_t>(chunks) * len * sizeof(double)));
  if (!partial) return TRL_ENOMEM;
  launch(k_block_dot_bulk<T, BS, JC, S, TB>, dim3(gj, static_cast<unsigned>(chunks)), kThreads, smem, h->stream, V, n * BS, nblk, W, n, rows_per_cta, partial, h->d_status, cond);
  int st = after_launch(h, "block_dot");
  if (st) return st;
  launch_reduce(h->stream, partial, chunks, len, C, cond);
  return after_launch(h, "block_dot reduce");
}

// Bulk-copy pipeline when a row of the block is a whole number of 16-byte units; otherwise
// the register-prefetch kernel with JC blocks and G row groups per warp iteration (about
// 16-20 independent loads in flight per warp).
template <typename T, int BS>
int launch_block_dot(trl_cuda_context* h, const T* V, int nblk, const T* W, int64_t n, double* C, const int* cond = nullptr)
{
  if (n == 0 && !cond) {
    cudaMemsetAsync(C, 0, static_cast<size_t>(nblk) * BS * BS * sizeof(double), h->stream);
    return TRL_OK;
  }
  // Shapes measured on B200 for the 884,736 x 8 blocks of the 96^3 workload (GB/s of
  // algorithmic bytes; the STREAM copy reference is 6,552): FP64 with 2 KB tiles, JC=8, S=3
  // gives 6,662 (24 blocks) and 6,970 (48 blocks); FP32 with 4 KB tiles gives 4,371 (8),
  // 5,269 (24) and with JC=4 5,804 (48).
  // A single block (the driver's T_ii = V_i^T W, both operands usually still in L2 from the
  // SpMM): the register-fed kernel with 8 (FP64) / 4 (FP32) row groups per warp and 4 CTAs
  // per SM measured 6,851 / 5,682 GB/s against 4,759 / 4,562 for the bulk pipeline.
  if (nblk == 1 && BS <= 8) return launch_block_dot_jc<T, BS, 1, (sizeof(T) == 8 ? 8 : 4)>(h, V, nblk, W, n, C, cond);
  if constexpr ((BS * sizeof(T)) % 16 == 0) {
    constexpr int TBS = (BS * sizeof(T) <= 64) ? 2048 : 4096; // small tiles where 32 rows fit
    constexpr int JCL = BS >= 16 ? 4 : 8;
    if (nblk == 1) return launch_block_dot_bulk<T, BS, 1, 8, 4096>(h, V, nblk, W, n, C, cond);
    if (nblk == 2) return launch_block_dot_bulk<T, BS, 2, 6, 4096>(h, V, nblk, W, n, C, cond);
    if (nblk <= 4) return launch_block_dot_bulk<T, BS, 4, 4, 4096>(h, V, nblk, W, n, C, cond);
    if constexpr (sizeof(T) == 8) return launch_block_dot_bulk<T, BS, JCL, 3, TBS>(h, V, nblk, W, n, C, cond);
    if (nblk <= 8) return launch_block_dot_bulk<T, BS, JCL, 3, 4096>(h, V, nblk, W, n, C, cond);
    return launch_block_dot_bulk<T, BS, 4, 3, TBS>(h, V, nblk, W, n, C, cond);
  }
  if (nblk == 1) return launch_block_dot_jc<T, BS, 1, 8>(h, V, nblk, W, n, C, cond);
  if (nblk == 2) return launch_block_dot_jc<T, BS, 2, 4>(h, V, nblk, W, n, C, cond);
  if (nblk <= 4) return launch_block_dot_jc<T, BS, 4, (BS >= 16 ? 2 : 4)>(h, V, nblk, W, n, C, cond);
  return launch_block_dot_jc<T, BS, (BS >= 16 ? 4 : 8), 2>(h, V, nblk, W, n, C, cond);
}

// Launches k_update_gram; the per-CTA Gram partial sums are left in the workspace
// (*partial, *chunks) for the caller to reduce.
template <typename T, int BS>
int launch_update_gram_partials(trl_cuda_context* h, const T* in, int MB, const double* coef, T* out, int64_t n, int accumulate, double sign, const int* cond,
                                double** partial, int* chunks)
{
  constexpr int NT = (BS + 7) / 8;
  // Measured on B200 (24 blocks of 884,736 x 8, GB/s of algorithmic bytes; copy peak
  // 6,539): one input block per loop iteration (U = 1) beats explicit multi-block register
  // prefetch (U = 4: FP64 6,075, FP32 3,860), and 8-row tiles per warp RT = 4 (FP64, 6,784)
  // and RT = 2 (FP32, 5,439) with two resident waves of CTAs do best.
  constexpr int RT = NT >= 2 ? 1 : (sizeof(T) == 8 ? 4 : 2);
  static int resident = 0;
  if (resident == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_update_gram<T, BS, RT, 1>, kThreads, 0) != cudaSuccess || resident < 1) resident = 4;
    cudaGetLastError();
  }
  const unsigned grid = grid_for(h, (n + 8 * RT - 1) / (8 * RT), kWarps, 2 * resident);
  *partial = static_cast<double*>(workspace(h, static_cast<size_t>(grid) * BS * BS * sizeof(double)));
  *chunks = static_cast<int>(grid);
  if (!*partial) return TRL_ENOMEM;
  launch(k_update_gram<T, BS, RT, 1>, grid, kThreads, 0, h->stream, in, n * BS, MB, coef, out, n, accumulate, sign, *partial, cond);
  return after_launch(h, "update_gram");
}

template <typename T, int BS>
int launch_update_gram(trl_cuda_context* h, const T* in, int MB, const double* coef, T* out, int64_t n, int accumulate, double sign, double* G, const int* cond)
{
  double* partial = nullptr;
  int chunks = 0;
  int st = launch_update_gram_partials<T, BS>(h, in, MB, coef, out, n, accumulate, sign, cond, &partial, &chunks);
  if (st) return st;
  launch_reduce(h->stream, partial, chunks, BS * BS, G, cond);
  return after_launch(h, "update_gram reduce");
}

template <typename T, int BS, int NBMAX>
void launch_gemm_nb(trl_cuda_context* h, const T* in, int MB, const double* coef, int ldc, int transpose, T* out, int nb, int64_t n, int accumulate, double sign)
{
  constexpr int NT = (BS + 7) / 8;
  constexpr int KS = (BS + 3) / 4;
  constexpr int RT = (NBMAX * NT >= 8) ? 1 : 2; // keep the accumulators within ~64 registers
  constexpr int U = (KS >= 4) ? 2 : 4;
  const unsigned grid = grid_for(h, (n + 8 * RT - 1) / (8 * RT), kWarps, 8);
  if (MB == 1) // a single input block: no point loading it U times
    launch(k_block_gemm<T, BS, NBMAX, RT, 1>, grid, kThreads, 0, h->stream, in, n * BS, MB, coef, ldc, transpose, out, n * BS, nb, n, accumulate, sign);
  else
    launch(k_block_gemm<T, BS, NBMAX, RT, U>, grid, kThreads, 0, h->stream, in, n * BS, MB, coef, ldc, transpose, out, n * BS, nb, n, accumulate, sign);
}

template <typename T, int BS>
int launch_block_gemm(trl_cuda_context* h, const T* in, int MB, const double* coef, int ldc, int transpose, T* out, int NB, int64_t n, int accumulate, double sign)
{
  if (n == 0 || NB == 0) return TRL_OK;
  constexpr int NBCAP = (BS >= 16) ? 4 : 16;
  for (int j0 = 0; j0 < NB; j0 += NBCAP) {
    const int nb = (NB - j0) < NBCAP ? (NB - j0) : NBCAP;
    const double* cj = coef + static_cast<int64_t>(j0) * BS * BS;
    T* oj = out + static_cast<int64_t>(j0) * n * BS;
    if (nb == 1)
      launch_gemm_nb<T, BS, 1>(h, in, MB, cj, ldc, transpose, oj, nb, n, accumulate, sign);
    else if (nb <= 2)
      launch_gemm_nb<T, BS, 2>(h, in, MB, cj, ldc, transpose, oj, nb, n, accumulate, sign);
    else if (nb <= 4)
      launch_gemm_nb<T, BS, 4>(h, in, MB, cj, ldc, transpose, oj, nb, n, accumulate, sign);
    else if (nb <= 8)
      launch_gemm_nb<T, BS, 8>(h, in, MB, cj, ldc, transpose, oj, nb, n, accumulate, sign);
    else
      launch_gemm_nb<T, BS, NBCAP>(h, in, MB, cj, ldc, transpose, oj, nb, n, accumulate, sign);
    int st = after_launch(h, "block_gemm");
    if (st) return st;
  }
  return TRL_OK;
}


// Restart rotation through k_rotate: the output columns are processed in chunks of at most 6
// n-tiles whose Yhat fragments fit in shared memory. Returns -1 (nothing launched) for block
// sizes below 4 or bases too deep for one k-step column of fragments; the caller then uses
// k_block_gemm.
template <typename T, int BS, int NTC>
int launch_rotate_chunk(trl_cuda_context* h, const T* V, int m, const double* Y, int ldy, int N, int c0, T* W, int64_t n, size_t smem)
{
  constexpr int RT = 2;
  constexpr int D = (BS >= 16) ? 2 : (BS == 8 ? 4 : 8);
  auto kern = k_rotate<T, BS, NTC, RT, D>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
    return set_error(h, TRL_ECUDA, "rotation: %zu bytes of shared memory refused", smem);
  const int64_t tiles = (n + 8 * RT - 1) / (8 * RT);
  int64_t grid = h->num_sms;
  const int64_t need = (tiles + kRotThreads / 32 - 1) / (kRotThreads / 32);
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  launch(kern, static_cast<unsigned>(grid), kRotThreads, smem, h->stream, V, n * BS, m, Y, ldy, N, c0, W, n * BS, n);
  return after_launch(h, "rotate");
}

template <typename T, int BS>
int launch_rotate(trl_cuda_context* h, const T* V, int m, const double* Y, int ldy, int k, T* W, int64_t n)
{
  if constexpr (BS < 4) {
    return -1;
  }
  else {
    constexpr size_t kSmemMax = 200 * 1024;
    const size_t frag_bytes = static_cast<size_t>(m) * (BS / 4) * 32 * sizeof(double); // one n-tile column
    int ntc_max = static_cast<int>(kSmemMax / frag_bytes);
    if (ntc_max > 6) ntc_max = 6; // beyond 6 n-tiles the accumulators spill at 128 registers
    if (ntc_max < 1) return -1;
    const int N = k * BS;
    const int tiles = (N + 7) / 8;
    const int passes = (tiles + ntc_max - 1) / ntc_max;
    const int per = (tiles + passes - 1) / passes;
    for (int t0 = 0; t0 < tiles; t0 += per) {
      const int ntc = (tiles - t0) < per ? (tiles - t0) : per;
      const size_t smem = frag_bytes * ntc;
      int st = TRL_OK;
      switch (ntc) {
      case 1: st = launch_rotate_chunk<T, BS, 1>(h, V, m, Y, ldy, N, t0 * 8, W, n, smem); break;
      case 2: st = launch_rotate_chunk<T, BS, 2>(h, V, m, Y, ldy, N, t0 * 8, W, n, smem); break;
      case 3: st = launch_rotate_chunk<T, BS, 3>(h, V, m, Y, ldy, N, t0 * 8, W, n, smem); break;
      case 4: st = launch_rotate_chunk<T, BS, 4>(h, V, m, Y, ldy, N, t0 * 8, W, n, smem); break;
      case 5: st = launch_rotate_chunk<T, BS, 5>(h, V, m, Y, ldy, N, t0 * 8, W, n, smem); break;
      default: st = launch_rotate_chunk<T, BS, 6>(h, V, m, Y, ldy, N, t0 * 8, W, n, smem); break;
      }
      if (st) return st;
    }
    return TRL_OK;
  }
}

} // namespace trl_detail

static int check_common(trl_cuda_context* h, int dtype, int64_t n, int bs)
{
  if (!valid_dtype(dtype)) return set_error(h, TRL_ENOTSUP, "unsupported dtype %d", dtype);
  if (!valid_bs(bs)) return set_error(h, TRL_ENOTSUP, "unsupported block size %d", bs);
  if (n < 0) return set_error(h, TRL_EINVAL, "negative row count");
  return TRL_OK;
}

static size_t elt_size(int dtype) { return dtype == TRL_F64 ? sizeof(double) : sizeof(float); }

extern "C" {

int trl_cuda_bv_zero(trl_cuda_handle h, int dtype, void* X, int64_t n, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  ProfScope prof(h, PROF_COPY, static_cast<double>(n) * bs * elt_size(dtype));
  return trl_cuda_memset_zero(h, X, static_cast<size_t>(n) * bs * elt_size(dtype));
}

int trl_cuda_bv_copy(trl_cuda_handle h, int dtype, void* X, const void* Y, int64_t n, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (X == Y) return TRL_OK;
  ProfScope prof(h, PROF_COPY, 2.0 * n * bs * elt_size(dtype));
  return trl_cuda_memcpy(h, X, Y, static_cast<size_t>(n) * bs * elt_size(dtype), TRL_D2D);
}

int trl_cuda_bv_sub(trl_cuda_handle h, int dtype, void* X, const void* Y, int64_t n, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  const int64_t count = n * bs;
  if (count == 0) return TRL_OK;
  if (!X || !Y) return set_error(h, TRL_EINVAL, "null pointer");
  ProfScope prof(h, PROF_SUB, 3.0 * count * elt_size(dtype));
  const int vec_ok = ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 15) == 0;
  const unsigned grid = grid_for(h, count / 4 + 1, kThreads, 8);
  TRL_DISPATCH_DT(dtype, launch(k_sub<T>, grid, kThreads, 0, h->stream, static_cast<T*>(X), static_cast<const T*>(Y), count, vec_ok));
  return after_launch(h, "bv_sub");
}

int trl_cuda_convert(trl_cuda_handle h, int dst_dtype, void* dst, int src_dtype, const void* src, int64_t count)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_dtype(dst_dtype) || !valid_dtype(src_dtype)) return set_error(h, TRL_ENOTSUP, "unsupported dtype");
  if (count < 0) return set_error(h, TRL_EINVAL, "negative count");
  if (count == 0) return TRL_OK;
  if (!dst || !src) return set_error(h, TRL_EINVAL, "null pointer");
  ProfScope prof(h, PROF_COPY, static_cast<double>(count) * (elt_size(dst_dtype) + elt_size(src_dtype)));
  if (dst_dtype == src_dtype) return trl_cuda_memcpy(h, dst, src, static_cast<size_t>(count) * elt_size(dst_dtype), TRL_D2D);
  const unsigned grid = grid_for(h, count, kThreads * 4, 8);
  if (dst_dtype == TRL_F64)
    launch(k_convert<double, float>, grid, kThreads, 0, h->stream, static_cast<double*>(dst), static_cast<const float*>(src), count);
  else
    launch(k_convert<float, double>, grid, kThreads, 0, h->stream, static_cast<float*>(dst), static_cast<const double*>(src), count);
  return after_launch(h, "convert");
}

int trl_cuda_bv_mult(trl_cuda_handle h, int dtype, int mode, const void* X, const double* W, void* Y, int64_t n, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (n == 0) return TRL_OK;
  if (!X || !W || !Y) return set_error(h, TRL_EINVAL, "null pointer");
  int transpose = 0, accumulate = 0;
  double sign = 1.0;
  switch (mode) {
  case TRL_MULT: break;
  case TRL_MULT_TRANSPOSE: transpose = 1; break;
  case TRL_MULT_ADD: accumulate = 1; break;
  case TRL_SUBTRACT:
    accumulate = 1;
    sign = -1.0;
    break;
  case TRL_SUBTRACT_TRANSPOSE:
    accumulate = 1;
    sign = -1.0;
    transpose = 1;
    break;
  default: return set_error(h, TRL_EINVAL, "bad mult mode %d", mode);
  }
  if (X == Y && accumulate) return set_error(h, TRL_EINVAL, "accumulating mult requires distinct input and output");
  ProfScope prof(h, PROF_MULT, (accumulate ? 3.0 : 2.0) * n * bs * elt_size(dtype), 2.0 * n * bs * bs);
  int st = TRL_OK;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, st = launch_block_gemm<T, BS>(h, static_cast<const T*>(X), 1, W, 1, transpose, static_cast<T*>(Y), 1, n, accumulate, sign)));
  return st;
}

int trl_cuda_block_dot(trl_cuda_handle h, int dtype, const void* V, int nblk, const void* W, int64_t n, int bs, double* C)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (nblk <= 0) return set_error(h, TRL_EINVAL, "nblk must be positive");
  if (!C) return set_error(h, TRL_EINVAL, "null pointer");
  if (n == 0) return trl_cuda_memset_zero(h, C, sizeof(double) * nblk * bs * bs); // empty sum
  if (!V || !W) return set_error(h, TRL_EINVAL, "null pointer");
  ProfScope prof(h, PROF_DOT, (nblk + 1.0) * n * bs * elt_size(dtype), 2.0 * nblk * n * bs * bs);
  int st = TRL_OK;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, st = launch_block_dot<T, BS>(h, static_cast<const T*>(V), nblk, static_cast<const T*>(W), n, C)));
  return st;
}

int trl_cuda_block_update(trl_cuda_handle h, int dtype, void* W, const void* V, int nblk, const double* C, int64_t n, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (nblk <= 0) return set_error(h, TRL_EINVAL, "nblk must be positive");
  if (n == 0) return TRL_OK;
  if (!V || !W || !C) return set_error(h, TRL_EINVAL, "null pointer");
  ProfScope prof(h, PROF_UPDATE, (nblk + 2.0) * n * bs * elt_size(dtype), 2.0 * nblk * n * bs * bs);
  int st = TRL_OK;
  // Coef(i, 0) = C + i*bs*bs  ->  ldc = 1
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, st = launch_block_gemm<T, BS>(h, static_cast<const T*>(V), nblk, C, 1, 0, static_cast<T*>(W), 1, n, 1, -1.0)));
  return st;
}

int trl_cuda_block_rotate(trl_cuda_handle h, int dtype, const void* V, int m, const double* Y, int ldy, int k, void* W, int64_t n, int bs)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (m <= 0 || k <= 0 || ldy < k) return set_error(h, TRL_EINVAL, "bad rotation shape m=%d k=%d ldy=%d", m, k, ldy);
  if (n == 0) return TRL_OK;
  if (!V || !Y || !W) return set_error(h, TRL_EINVAL, "null pointer");
  const size_t es = elt_size(dtype);
  const char* v0 = static_cast<const char*>(V);
  const char* v1 = v0 + static_cast<size_t>(m) * n * bs * es;
  const char* w0 = static_cast<const char*>(W);
  const char* w1 = w0 + static_cast<size_t>(k) * n * bs * es;
  if (w0 < v1 && v0 < w1) return set_error(h, TRL_EINVAL, "rotation output overlaps its input");
  ProfScope prof(h, PROF_ROTATE, (static_cast<double>(m) + k) * n * bs * es, 2.0 * n * m * k * bs * bs);
  int st = TRL_OK;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, {
    st = launch_rotate<T, BS>(h, static_cast<const T*>(V), m, Y, ldy, k, static_cast<T*>(W), n);
    if (st == -1) st = launch_block_gemm<T, BS>(h, static_cast<const T*>(V), m, Y, ldy, 0, static_cast<T*>(W), k, n, 0, 1.0);
  }));
  return st;
}

int trl_cuda_cholqr(trl_cuda_handle h, int dtype, void* X, int64_t n, int bs, int passes, double* R)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (passes < 1 || passes > 4) return set_error(h, TRL_EINVAL, "passes must be in [1, 4]");
  if (!X || !R) return set_error(h, TRL_EINVAL, "null pointer");
  double* small = static_cast<double*>(small_scratch(h));
  if (!small) return TRL_ENOMEM;
  double* G = small;
  ProfScope prof(h, PROF_CHOLQR, 3.0 * passes * n * bs * elt_size(dtype), 4.0 * passes * n * bs * bs);
  int st = trl_cuda_block_dot(h, dtype, X, 1, X, n, bs, G);
  if (st) return st;
  return trl_cuda_cholqr_gram(h, dtype, X, n, bs, passes, R, G);
}

// Per pass: one-CTA factor of the Gram matrix, then the apply X <- X U^{-1}, which also
// forms the partial Gram sums of the result for the next pass's factor.
int trl_cuda_cholqr_gram(trl_cuda_handle h, int dtype, void* X, int64_t n, int bs, int passes, double* R, const double* G0)
{
  TRL_CHECK_HANDLE(h);
  if (!G0) return trl_cuda_cholqr(h, dtype, X, n, bs, passes, R);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (passes < 1 || passes > 4) return set_error(h, TRL_EINVAL, "passes must be in [1, 4]");
  if (!X || !R) return set_error(h, TRL_EINVAL, "null pointer");
  double* small = static_cast<double*>(small_scratch(h));
  if (!small) return TRL_ENOMEM;
  double* Uinv = small + 256;
  double* gsum = small + 512;                                // the factor's reduced Gram entries
  unsigned* ticket = reinterpret_cast<unsigned*>(small + 768); // zero between launches
  ProfScope prof(h, PROF_CHOLQR, 2.0 * passes * n * bs * elt_size(dtype), 4.0 * passes * n * bs * bs);
  const double* src = G0; // the Gram matrix, or per-CTA partial sums of it
  int chunks = 0;
  for (int p = 0; p < passes; ++p) {
    int st = TRL_OK;
    TRL_DISPATCH_BS(bs, launch(k_gram_factor<BS>, chunks > 0 ? static_cast<unsigned>((BS * BS + kFactorOPC - 1) / kFactorOPC) : 1u, kRedThreads, 0, h->stream, src, chunks,
                               Uinv, R, p == 0, h->d_status, gsum, ticket));
    st = after_launch(h, "cholqr factor");
    if (st) return st;
    if (p + 1 < passes) {
      double* partial = nullptr;
      TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, st = launch_update_gram_partials<T, BS>(h, static_cast<const T*>(X), 1, Uinv, static_cast<T*>(X), n, 0, 1.0, nullptr, &partial, &chunks)));
      src = partial;
    }
    else {
      TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, st = launch_block_gemm<T, BS>(h, static_cast<const T*>(X), 1, Uinv, 1, 0, static_cast<T*>(X), 1, n, 0, 1.0)));
    }
    if (st) return st;
  }
  return TRL_OK;
}

int trl_cuda_project_out(trl_cuda_handle h, int dtype, const void* V, int nblk, void* W, int64_t n, int bs, int mode, double eta, double* G)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (nblk <= 0 || !G) return set_error(h, TRL_EINVAL, "bad project_out arguments");
  if (mode != TRL_CGS_ONE && mode != TRL_CGS_TWO && mode != TRL_CGS_IFNEEDED) return set_error(h, TRL_EINVAL, "bad project_out mode %d", mode);
  const int BB = bs * bs;
  if (n == 0) return trl_cuda_memset_zero(h, G, sizeof(double) * BB);
  if (!V || !W) return set_error(h, TRL_EINVAL, "null pointer");
  const size_t es = elt_size(dtype);
  // coefficient storage: C1 (nblk+1 blocks) | C2 (nblk blocks) | Gw0 | Gw1 | Gw2 | flag
  double* base = static_cast<double*>(workspace2(h, sizeof(double) * (static_cast<size_t>(2 * nblk + 4) * BB) + 64));
  if (!base) return TRL_ENOMEM;
  double* C1 = base;
  double* C2 = C1 + static_cast<size_t>(nblk + 1) * BB;
  double* Gw0 = C2 + static_cast<size_t>(nblk) * BB;
  double* Gw1 = Gw0 + BB;
  double* Gw2 = Gw1 + BB;
  int* flag = reinterpret_cast<int*>(Gw2 + BB);
  const bool contiguous = static_cast<const char*>(W) == static_cast<const char*>(V) + static_cast<size_t>(nblk) * n * bs * es;
  int st = TRL_OK;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, {
    const T* Vt = static_cast<const T*>(V);
    T* Wt = static_cast<T*>(W);
    // pass 1: C1 = V^T w (and w^T w, for free when w is the block right after V)
    {
      ProfScope prof(h, PROF_DOT, (nblk + (contiguous ? 1.0 : 2.0)) * n * bs * es, 2.0 * (nblk + 1) * n * bs * bs);
      if (contiguous) {
        st = launch_block_dot<T, BS>(h, Vt, nblk + 1, Wt, n, C1);
        if (!st) st = trl_cuda_memcpy(h, Gw0, C1 + static_cast<size_t>(nblk) * BB, sizeof(double) * BB, TRL_D2D);
      }
      else {
        st = launch_block_dot<T, BS>(h, Vt, nblk, Wt, n, C1);
        if (!st) st = launch_block_dot<T, BS>(h, Wt, 1, Wt, n, Gw0);
      }
    }
    if (st) return st;
    {
      ProfScope prof(h, PROF_UPDATE, (nblk + 2.0) * n * bs * es, 2.0 * nblk * n * bs * bs + 2.0 * n * bs * bs);
      st = launch_update_gram<T, BS>(h, Vt, nblk, C1, Wt, n, 1, -1.0, Gw1, nullptr);
    }
    if (st) return st;
    if (mode == TRL_CGS_ONE) return trl_cuda_memcpy(h, G, Gw1, sizeof(double) * BB, TRL_D2D);
    if (mode == TRL_CGS_TWO) {
      cudaMemsetAsync(flag, 0x01, sizeof(int), h->stream);
    }
    else {
      launch(k_dgks_flag<BS>, 1, 32, 0, h->stream, Gw0, Gw1, eta * eta, flag);
      if ((st = after_launch(h, "dgks"))) return st;
    }
    // pass 2, only where the flag is set (decided on the device; its bytes are not credited
    // to the profile because the host does not know whether it ran)
    {
      ProfScope prof(h, PROF_REORTH2, 0.0);
      st = launch_block_dot<T, BS>(h, Vt, nblk, Wt, n, C2, flag);
      if (!st) st = launch_update_gram<T, BS>(h, Vt, nblk, C2, Wt, n, 1, -1.0, Gw2, flag);
    }
    if (st) return st;
    launch(k_select_block, 1, 256, 0, h->stream, flag, Gw2, Gw1, G, BB);
    st = after_launch(h, "select");
  }));
  return st;
}

int trl_cuda_project_out_sketch(trl_cuda_handle h, int dtype, const void* V, int nblk, void* W, int64_t n, int bs, const void* S, double thr, double eta, double* G,
                                int* pair_state)
{
  TRL_CHECK_HANDLE(h);
  if (int st = check_common(h, dtype, n, bs)) return st;
  if (nblk <= 0 || !G || !(thr >= 0.0)) return set_error(h, TRL_EINVAL, "bad project_out_sketch arguments");
  const int BB = bs * bs;
  if (n == 0) return trl_cuda_memset_zero(h, G, sizeof(double) * BB);
  if (!V || !W || !S) return set_error(h, TRL_EINVAL, "null pointer");
  // coefficient storage: C1 (nblk blocks) | C2 (nblk blocks) | E | Gw0 | Gw1 | Gw2 | flags
  double* base = static_cast<double*>(workspace2(h, sizeof(double) * (static_cast<size_t>(2 * nblk + 4) * BB) + 64));
  if (!base) return TRL_ENOMEM;
  double* C1 = base;
  double* C2 = C1 + static_cast<size_t>(nblk) * BB;
  double* E = C2 + static_cast<size_t>(nblk) * BB; // [E; Gw0] = [S, W]^T W in one pass
  double* Gw0 = E + BB;
  double* Gw1 = Gw0 + BB;
  double* Gw2 = Gw1 + BB;
  int* flag1 = reinterpret_cast<int*>(Gw2 + BB);
  int* flag2 = flag1 + 1;
  const size_t es = elt_size(dtype);
  int st = TRL_OK;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, {
    const T* Vt = static_cast<const T*>(V);
    const T* St = static_cast<const T*>(S);
    T* Wt = static_cast<T*>(W);
    {
      ProfScope prof(h, PROF_DOT, 3.0 * n * bs * es, 4.0 * n * bs * bs);
      st = launch_block_dot_two<T, BS>(h, St, Wt, Wt, n, E);
    }
    if (st) return st;
    launch(k_sketch_flag<BS>, 1, 32, 0, h->stream, E, Gw0, thr * thr, flag1, pair_state);
    if ((st = after_launch(h, "sketch flag"))) return st;
    // both passes only where flagged (decided on the device; their bytes are not credited
    // to the profile because the host does not know whether they ran)
    {
      ProfScope prof(h, PROF_REORTH2, 0.0);
      st = launch_block_dot<T, BS>(h, Vt, nblk, Wt, n, C1, flag1);
      if (!st) st = launch_update_gram<T, BS>(h, Vt, nblk, C1, Wt, n, 1, -1.0, Gw1, flag1);
      if (st) return st;
      launch(k_dgks_flag_after<BS>, 1, 32, 0, h->stream, flag1, Gw0, Gw1, eta * eta, flag2);
      if ((st = after_launch(h, "dgks"))) return st;
      st = launch_block_dot<T, BS>(h, Vt, nblk, Wt, n, C2, flag2);
      if (!st) st = launch_update_gram<T, BS>(h, Vt, nblk, C2, Wt, n, 1, -1.0, Gw2, flag2);
    }
    if (st) return st;
    launch(k_select_block3, 1, 256, 0, h->stream, flag1, flag2, Gw0, Gw1, Gw2, G, BB);
    st = after_launch(h, "select");
#ifdef TRL_DEBUG_TRACE
    // debug builds (-DTRL_DEBUG_TRACE) with TRL_PARTIAL_TRACE set: one stderr line per call
    // (synchronises; diagnostics only)
    static const bool trace = std::getenv("TRL_PARTIAL_TRACE") != nullptr;
    if (!st && trace) {
      double eg[2 * 256];
      int fl[2];
      cudaMemcpyAsync(eg, E, sizeof(double) * 2 * BB, cudaMemcpyDeviceToHost, h->stream);
      cudaMemcpyAsync(fl, flag1, sizeof(int) * 2, cudaMemcpyDeviceToHost, h->stream);
      cudaStreamSynchronize(h->stream);
      double e2 = 0.0, tr = 0.0;
      for (int i = 0; i < BB; ++i) e2 += eg[i] * eg[i];
      for (int c = 0; c < bs; ++c) tr += eg[BB + c * bs + c];
      std::fprintf(stderr, "partial nblk %d loss %.3e projected %d forced %d second %d\n", nblk, std::sqrt(e2 / tr), fl[0] & 1, (fl[0] >> 1) & 1, fl[1]);
    }
#endif
  }));
  return st;
}

} // extern "C"

namespace {
__global__ void __launch_bounds__(kThreads) k_unblock(const double* __restrict__ X, int64_t n, int bs, int ncols, double* __restrict__ out)
{
  ::trl_detail::pdl_enter();
  const int64_t total = n * ncols;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int64_t r = e / ncols;
    const int c = static_cast<int>(e % ncols);
    out[e] = X[static_cast<int64_t>(c / bs) * n * bs + r * bs + (c % bs)];
  }
}
} // namespace

extern "C" int trl_cuda_unblock(trl_cuda_handle h, const double* X, int64_t n, int bs, int ncols, double* out)
{
  TRL_CHECK_HANDLE(h);
  if (!valid_bs(bs) || n < 0 || ncols < 0) return set_error(h, TRL_EINVAL, "bad unblock arguments");
  if (n == 0 || ncols == 0) return TRL_OK;
  if (!X || !out) return set_error(h, TRL_EINVAL, "null pointer");
  ProfScope prof(h, PROF_COPY, 16.0 * n * ncols);
  launch(k_unblock, grid_for(h, n * ncols, kThreads * 4, 8), kThreads, 0, h->stream, X, n, bs, ncols, out);
  return after_launch(h, "unblock");
}

// ---------------------------------------------------------------- allocation-free block dot
// trl_cuda_block_dot_noalloc: the multi-block inner product for callers that must not
// allocate device memory. Its per-chunk partial sums live in the fixed array below instead
// of a handle's workspace. One copy of the array (2 MiB) exists on every GPU that loads this
// library and stays there until the process exits.
#include <mutex>

static constexpr int64_t kNoAllocScratchDoubles = int64_t(1) << 18; // 2 MiB of FP64 partials
static constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocScratchDoubles];

static std::mutex g_noalloc_mutex;
static double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
static int g_noalloc_sms[kNoAllocMaxDevices] = {};

// Resolves the device address of the scratch array on the current device (once per device).
static int noalloc_scratch(int device, double** ptr, int* sms)
{
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return TRL_ECUDA;
    }
    int count = 0;
    if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || count <= 0) {
      cudaGetLastError();
      return TRL_ECUDA;
    }
    g_noalloc_sms[device] = count;
    g_noalloc_ptr[device] = static_cast<double*>(p);
  }
  *ptr = g_noalloc_ptr[device];
  *sms = g_noalloc_sms[device];
  return TRL_OK;
}

template <typename T, int BS, int JC, int G>
static int noalloc_dot(cudaStream_t stream, int sms, double* partial, const T* V, int nblk, const T* W, int64_t n, double* C)
{
  const int64_t len = static_cast<int64_t>(nblk) * BS * BS;
  const int gj = (nblk + JC - 1) / JC;
  int64_t chunks = static_cast<int64_t>(sms) * 4 / gj;
  const int64_t fit = kNoAllocScratchDoubles / len; // chunks whose partials fit the array
  if (chunks > fit) chunks = fit;
  const int64_t max_chunks = (n + 511) / 512;
  if (chunks > max_chunks) chunks = max_chunks;
  if (chunks < 1) chunks = 1;
  int64_t rows_per_cta = (n + chunks - 1) / chunks;
  constexpr int step = kWarps * 4 * G;
  rows_per_cta = (rows_per_cta + step - 1) / step * step;
  chunks = (n + rows_per_cta - 1) / rows_per_cta;
  // every (chunk, block) entry of the partials is written before it is read in this call,
  // so nothing left in the array by an earlier call is used and nothing needs clearing
  launch(k_block_dot<T, BS, JC, G>, dim3(gj, static_cast<unsigned>(chunks)), kThreads, 0, stream, V, n * BS, nblk, W, n, rows_per_cta, partial, nullptr);
  if (cudaGetLastError() != cudaSuccess) return TRL_ECUDA;
  launch_reduce(stream, partial, chunks, len, C, nullptr);
  if (cudaGetLastError() != cudaSuccess) return TRL_ECUDA;
  return TRL_OK;
}

template <typename T, int BS>
static int noalloc_dot_dispatch(cudaStream_t stream, int sms, double* partial, const T* V, int nblk, const T* W, int64_t n, double* C)
{
  if (nblk == 1) return noalloc_dot<T, BS, 1, 8>(stream, sms, partial, V, nblk, W, n, C);
  if (nblk == 2) return noalloc_dot<T, BS, 2, 4>(stream, sms, partial, V, nblk, W, n, C);
  if (nblk <= 4) return noalloc_dot<T, BS, 4, (BS >= 16 ? 2 : 4)>(stream, sms, partial, V, nblk, W, n, C);
  return noalloc_dot<T, BS, (BS >= 16 ? 4 : 8), 2>(stream, sms, partial, V, nblk, W, n, C);
}

extern "C" int trl_cuda_block_dot_noalloc(void* stream, int dtype, const void* V, int nblk, const void* W, int64_t n, int bs, double* C)
{
  if (!valid_dtype(dtype) || !valid_bs(bs)) return TRL_ENOTSUP;
  if (nblk <= 0 || n < 0 || !C) return TRL_EINVAL;
  if (static_cast<int64_t>(nblk) * bs * bs > TRL_CUDA_NOALLOC_MAX_ENTRIES) return TRL_EINVAL; // the output would not fit the partial-sum array
  auto s = static_cast<cudaStream_t>(stream);
  if (n == 0) return cudaMemsetAsync(C, 0, sizeof(double) * nblk * bs * bs, s) == cudaSuccess ? TRL_OK : TRL_ECUDA;
  if (!V || !W) return TRL_EINVAL;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kNoAllocMaxDevices) {
    cudaGetLastError();
    return TRL_ECUDA;
  }
  double* partial = nullptr;
  int sms = 0;
  if (int st = noalloc_scratch(device, &partial, &sms)) return st;
  int st = TRL_OK;
  trl_cuda_context* h = nullptr; // only for the dispatch macros' error path
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, st = noalloc_dot_dispatch<T, BS>(s, sms, partial, static_cast<const T*>(V), nblk, static_cast<const T*>(W), n, C)));
  return st;
}

namespace {

// FP64 tensor-core (DMMA m8n8k4) issue rate: every warp runs kDmmaChains independent
// accumulator chains for `iters` rounds; the result is written so that nothing is elided.
constexpr int kDmmaChains = 8;

__global__ void __launch_bounds__(256) k_dmma_rate(int iters, double* __restrict__ out)
{
  ::trl_detail::pdl_enter();
  double d0[kDmmaChains], d1[kDmmaChains];
  const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * blockIdx.x;
#pragma unroll
  for (int c = 0; c < kDmmaChains; ++c) d0[c] = d1[c] = 0.0;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int c = 0; c < kDmmaChains; ++c) dmma_m8n8k4(d0[c], d1[c], a, b);
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kDmmaChains; ++c) s += d0[c] + d1[c];
  if (s == 12345.678) out[0] = s; // never true; keeps the chains alive
}

} // namespace

extern "C" int trl_cuda_measure_dmma_rate(trl_cuda_handle h, double* host_tflops)
{
  TRL_CHECK_HANDLE(h);
  if (!host_tflops) return set_error(h, TRL_EINVAL, "null output");
  double* out = static_cast<double*>(small_scratch(h));
  if (!out) return TRL_ENOMEM;
  const int iters = 4096;
  const unsigned grid = static_cast<unsigned>(h->num_sms) * 8;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch(k_dmma_rate, grid, 256, 0, h->stream, iters, out); // warm-up
  cudaEventRecord(a, h->stream);
  launch(k_dmma_rate, grid, 256, 0, h->stream, iters, out);
  cudaEventRecord(b, h->stream);
  const cudaError_t e = cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "dmma rate: %s", cudaGetErrorString(e));
  if (int st = after_launch(h, "dmma rate")) return st;
  const double flops = 2.0 * 8 * 8 * 4 * kDmmaChains * static_cast<double>(iters) * grid * (256 / 32);
  *host_tflops = flops / (ms * 1e-3) / 1e12;
  return TRL_OK;
}
