// A prepared copy of a CSR operator for repeated SpMMs (trl_cuda_op_*): sliced ELLPACK with
// rows sorted by length inside windows (SELL-C-sigma, Kreutzer et al. 2014), and the SpMM
// Y_j = alpha*A*X_j + beta*X_j + gamma*W_j on it.
//
// Layout. Rows are sorted by decreasing length, stably, inside windows of kSellWindow rows
// (sigma); `perm[p]` is the original row at sorted position p (-1 past the last row).
// Slice s holds the C rows at sorted positions s*C .. s*C+C-1, padded to the slice's
// longest row; entry (slot j, row q) of slice s sits at sptr[s] + j*C + q, so one slot of
// a slice is C consecutive column indices and C consecutive values. Padding entries carry
// value 0 and a column the row already reads (its last one), so they add nothing and their
// gathers hit cached rows. C is the number of rows one warp covers per step of the SpMM for
// the operator's dtype and block size (RPW below), so a warp loads a slot's indices and
// values with one coalesced load each, straight into registers.
//
// Every row sums its entries in CSR order, whatever its position after the sort, so the
// results are bit-identical to the CSR kernel's per-row walk (trl_cuda_spmm_blocks).
#include "common.cuh"

#include <algorithm>
#include <cstring>

namespace {

using namespace trl_detail;

constexpr int kSellWindow = 4096; // sigma
constexpr int kSellKeys = 1024;   // sort keys: lengths >= kSellKeys - 2 share the first key
constexpr int kBuildThreads = 256;
constexpr int kBuildWarps = kBuildThreads / 32;
constexpr int kScanItems = 2048; // slices per CTA of the slice-pointer scan (256 threads x 8)

// Row mapping of the SpMM for element type T and block size BS: a row is owned by LPR
// lanes, each carrying VEC adjacent columns (32 bytes at most: one 256-bit load), so that
// one X row is one LPR-lane gather; a warp covers RPW = 32 / LPR rows, the slice height.
template <typename T, int BS>
struct SellShape {
  static constexpr int max_vec = 32 / static_cast<int>(sizeof(T));
  static constexpr int VEC = max_vec < BS ? max_vec : BS;
  static constexpr int LPR = BS / VEC;
  static constexpr int RPW = 32 / LPR;
};

// VEC adjacent elements (VEC * sizeof(T) <= 32 bytes, aligned to that size) through the
// read-only path; 32-byte vectors with one 256-bit load.
template <typename T, int VEC>
__device__ __forceinline__ void load_row(const T* p, T (&out)[VEC])
{
  if constexpr (VEC * sizeof(T) == 32) {
    if constexpr (sizeof(T) == 8)
      asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(out[0]), "=d"(out[1]), "=d"(out[2]), "=d"(out[3]) : "l"(p));
    else
      asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=f"(out[0]), "=f"(out[1]), "=f"(out[2]), "=f"(out[3]), "=f"(out[4]), "=f"(out[5]), "=f"(out[6]), "=f"(out[7])
                   : "l"(p));
  }
  else
    load_vec<T, VEC>(p, out);
}

template <typename T, int VEC>
__device__ __forceinline__ void store_row(T* p, const T (&in)[VEC])
{
  if constexpr (VEC * sizeof(T) == 32) {
    constexpr int H = VEC / 2;
    T lo[H], hi[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
      lo[i] = in[i];
      hi[i] = in[H + i];
    }
    store_vec<T, H>(p, lo);
    store_vec<T, H>(p + H, hi);
  }
  else
    store_vec<T, VEC>(p, in);
}

template <typename T>
int slice_height_for(int bs)
{
  switch (bs) {
  case 1: return SellShape<T, 1>::RPW;
  case 2: return SellShape<T, 2>::RPW;
  case 4: return SellShape<T, 4>::RPW;
  case 8: return SellShape<T, 8>::RPW;
  case 16: return SellShape<T, 16>::RPW;
  default: return 0;
  }
}

__device__ __forceinline__ int sort_key(int64_t r, int64_t n, const int32_t* __restrict__ rowptr)
{
  if (r >= n) return kSellKeys - 1; // past the last row: after every real row
  const int len = __ldg(rowptr + r + 1) - __ldg(rowptr + r);
  return (kSellKeys - 2) - min(len, kSellKeys - 2); // ascending key = descending length
}

// One warp per window: stable counting sort of the window's rows by key. perm has
// nwin * kSellWindow entries.
__global__ void __launch_bounds__(kBuildThreads) k_sell_sort(int64_t n, int64_t nwin, const int32_t* __restrict__ rowptr, int32_t* __restrict__ perm)
{
  ::trl_detail::pdl_enter();
  __shared__ int bins[kBuildWarps][kSellKeys];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t win = static_cast<int64_t>(blockIdx.x) * kBuildWarps + w;
  if (win >= nwin) return; // whole warp; the kernel has no CTA-wide barrier
  int* b = bins[w];
  for (int i = lane; i < kSellKeys; i += 32) b[i] = 0;
  __syncwarp();
  const int64_t r0 = win * kSellWindow;
  for (int t = 0; t < kSellWindow; t += 32) {
    const int key = sort_key(r0 + t + lane, n, rowptr);
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (lane == __ffs(peers) - 1) b[key] += __popc(peers);
    __syncwarp();
  }
  // exclusive scan of the counts, 32 consecutive keys per lane
  constexpr int PER = kSellKeys / 32;
  int loc[PER];
  int sum = 0;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    loc[q] = b[lane * PER + q];
    sum += loc[q];
  }
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  int run = incl - sum;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    b[lane * PER + q] = run;
    run += loc[q];
  }
  __syncwarp();
  // stable scatter: rows of one key keep their order (lane order within a step, steps in order)
  for (int t = 0; t < kSellWindow; t += 32) {
    const int64_t r = r0 + t + lane;
    const int key = sort_key(r, n, rowptr);
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int base = b[key];
    perm[r0 + base + rank] = r < n ? static_cast<int32_t>(r) : -1;
    __syncwarp();
    if (lane == __ffs(peers) - 1) b[key] = base + __popc(peers);
    __syncwarp();
  }
}

// Slice lengths (entries per row of the slice) and, per CTA of kScanItems slices, the
// inclusive scan of length * C into sptr[1 + s] (CTA-local) and the CTA's total into
// part[blockIdx.x]; the largest slice length into stats[1] (atomicMax).
__global__ void __launch_bounds__(256) k_sell_slices(int64_t nslices, int C, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ perm,
                                                     int64_t* __restrict__ sptr, int64_t* __restrict__ part, unsigned long long* __restrict__ stats)
{
  ::trl_detail::pdl_enter();
  constexpr int PER = kScanItems / 256;
  __shared__ int64_t warp_tot[8];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t s0 = static_cast<int64_t>(blockIdx.x) * kScanItems + static_cast<int64_t>(tid) * PER;
  int64_t v[PER];
  int64_t sum = 0;
  int longest = 0;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int64_t s = s0 + q;
    int len = 0;
    if (s < nslices)
      for (int i = 0; i < C; ++i) {
        const int r = perm[s * C + i];
        if (r >= 0) len = max(len, __ldg(rowptr + r + 1) - __ldg(rowptr + r));
      }
    longest = max(longest, len);
    v[q] = static_cast<int64_t>(len) * C;
    sum += v[q];
  }
  int64_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t x = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += x;
  }
  if (lane == 31) warp_tot[w] = incl;
  for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
  if (lane == 0 && longest > 0) atomicMax(&stats[1], static_cast<unsigned long long>(longest));
  __syncthreads();
  int64_t before = 0;
  for (int i = 0; i < w; ++i) before += warp_tot[i];
  int64_t run = before + incl - sum;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    run += v[q];
    if (s0 + q < nslices) sptr[1 + s0 + q] = run;
  }
  if (tid == 255) part[blockIdx.x] = before + incl;
}

// Exclusive scan of the per-CTA totals (one CTA, any count) in place; the grand total into
// stats[0]; sptr[0] = 0.
__global__ void __launch_bounds__(1024) k_sell_scan_parts(int64_t nparts, int64_t* __restrict__ part, int64_t* __restrict__ sptr, unsigned long long* __restrict__ stats)
{
  ::trl_detail::pdl_enter();
  __shared__ int64_t warp_tot[32];
  __shared__ int64_t carry;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nparts; base += 1024) {
    const int64_t i = base + tid;
    const int64_t x = i < nparts ? part[i] : 0;
    int64_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    int64_t before = carry;
    for (int q = 0; q < w; ++q) before += warp_tot[q];
    if (i < nparts) part[i] = before + incl - x;
    __syncthreads();
    if (tid == 1023) carry = before + incl;
    __syncthreads();
  }
  if (tid == 0) {
    sptr[0] = 0;
    stats[0] = static_cast<unsigned long long>(carry);
  }
}

__global__ void __launch_bounds__(256) k_sell_add_parts(int64_t nslices, const int64_t* __restrict__ part, int64_t* __restrict__ sptr)
{
  ::trl_detail::pdl_enter();
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s < nslices) sptr[1 + s] += part[s / kScanItems];
}

// One warp per slice: lane l covers row q = l % C of slots j0 + l / C.
template <typename V>
__global__ void __launch_bounds__(kBuildThreads) k_sell_fill(int64_t nslices, int C, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind,
                                                          const V* __restrict__ vals, const int32_t* __restrict__ perm, const int64_t* __restrict__ sptr,
                                                          int32_t* __restrict__ scol, V* __restrict__ sval)
{
  ::trl_detail::pdl_enter();
  const int lane = threadIdx.x & 31;
  const int64_t wstride = static_cast<int64_t>(gridDim.x) * kBuildWarps;
  const int q = lane % C, jj = lane / C, spj = 32 / C; // slots per warp step
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kBuildWarps + (threadIdx.x >> 5); s < nslices; s += wstride) {
    const int64_t e0 = sptr[s];
    const int slen = static_cast<int>((sptr[s + 1] - e0) / C);
    const int r = perm[s * C + q];
    const int rs = r >= 0 ? __ldg(rowptr + r) : 0;
    const int len = r >= 0 ? __ldg(rowptr + r + 1) - rs : 0;
    const int32_t pad_col = len > 0 ? __ldg(colind + rs + len - 1) : (r >= 0 ? r : 0);
    for (int j = jj; j < slen; j += spj) {
      const bool real = j < len;
      scol[e0 + static_cast<int64_t>(j) * C + q] = real ? __ldg(colind + rs + j) : pad_col;
      sval[e0 + static_cast<int64_t>(j) * C + q] = real ? vals[rs + j] : V(0);
    }
  }
}

} // namespace

namespace {

constexpr int kSpmmThreads = 256;
constexpr int kSpmmWarps = kSpmmThreads / 32;

// Per instantiation: NBG blocks accumulated per pass over a slice (1 for the single-block
// SpMM; the multi-block SpMM takes up to kSellBlocksPerPass blocks per pass and re-reads a
// slice's indices and values, from L2, for each further pass), UG slots per group, and the
// CTAs per SM the registers must allow.
template <typename T, int BS, int NBG, bool LONG>
struct SellTune {
  static constexpr int lane_bytes = SellShape<T, BS>::VEC * static_cast<int>(sizeof(T));
  static constexpr int ug = 64 / lane_bytes;
  // operators with long rows (LONG: 16 or more slots per slice on average) keep 8 slots of
  // gathers in flight per lane at two CTAs per SM; short rows prefer more warps with fewer
  // slots each (measured on B200: 96^3 stencil, 7 slots per slice, 0.56 of the copy peak
  // with 2 slots x 4 CTAs against 0.53 with 8 x 2; elasticity, 81 slots, 0.50 with 8 x 2
  // against 0.39 with 2 x 4). Several blocks per pass keep one slot per lane in flight for
  // each block.
  static constexpr int UG = NBG == 1 ? (LONG ? 8 : (ug > 4 ? 4 : ug)) : (NBG > 2 ? 1 : 2);
  static constexpr int MINB = NBG == 1 ? (LONG ? 2 : 4) : 2;
};

// Blocks per pass of the multi-block SpMM (the Chebyshev filter's kept blocks). Measured on
// B200 with 6 blocks of the 96^3 stencil, bs 8, behind an L2 flush (fraction of the copy
// peak, FP64 / FP32): 2 blocks x 2 slots per pass 0.40 / 0.40; 3 x 2: 0.49 / 0.47; 3 x 1 at 3
// CTAs per SM: 0.40 / 0.39; 4 x 1: 0.40 / 0.31; 6 x 1 (one pass, 128 registers, 2 CTAs per
// SM): 0.55 / 0.50.
constexpr int kSellBlocksPerPass = 6;

// Asks L2 to fetch [p, p + bytes) (a bulk prefetch: no registers, no shared memory). p and
// bytes are multiples of 16.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Warp per slice; lanes: grp = lane / LPR is the slice row, sub = lane % LPR the column
// chunk. Slices are taken in natural order, or (interleave) window-major within each slice
// rank so that the long first slices of all windows spread over all warps.
// The warp walks its slices as one stream of slot groups (UG slots of one slice each) and
// keeps one group ahead: while the gathers and value loads of group g are in flight it
// loads the column indices of group g + 1, which may belong to the next slice. The bounds
// and rows of the next slice are loaded one slice ahead, and lane 0 asks L2 for the slice
// after it (bulk prefetch), so that the index loads hit L2.
template <typename T, int BS, int NBG, bool LONG>
__global__ void __launch_bounds__(kSpmmThreads, SellTune<T, BS, NBG, LONG>::MINB)
    k_spmm_sell(int nslices, int nwin, int spw, int interleave, const int32_t* __restrict__ perm, const int64_t* __restrict__ sptr, const int32_t* __restrict__ scol,
                const T* __restrict__ sval, const T* __restrict__ X, T* Y, T alpha, T beta, T gamma, const T* W, int nb, int64_t bstride)
{
  ::trl_detail::pdl_enter();
  using S = SellShape<T, BS>;
  constexpr int VEC = S::VEC, LPR = S::LPR, C = S::RPW, UG = SellTune<T, BS, NBG, LONG>::UG;
  const int lane = threadIdx.x & 31;
  const int grp = lane / LPR, sub = lane % LPR;
  const int wstride = static_cast<int>(gridDim.x) * kSpmmWarps;
  const int total = interleave ? nwin * spw : nslices;
  auto slice_of = [&](int i) -> int {
    return interleave ? static_cast<int>(static_cast<unsigned>(i) % static_cast<unsigned>(nwin)) * spw + static_cast<int>(static_cast<unsigned>(i) / static_cast<unsigned>(nwin)) : i;
  };
  auto next_valid = [&](int i) { // next index at or after i whose slice exists (total if none)
    while (i < total && slice_of(i) >= nslices) i += wstride;
    return i;
  };
  struct Slice {
    int64_t e0, e1;
    int row;
  };
  auto load_slice = [&](int i) {
    Slice q{0, 0, -1};
    if (i < total) {
      const int s = slice_of(i);
      q.e0 = __ldg(sptr + s);
      q.e1 = __ldg(sptr + s + 1);
      q.row = __ldg(perm + static_cast<int64_t>(s) * C + grp);
    }
    return q;
  };
  auto prefetch_slice = [&](const Slice& q) {
    if (lane == 0 && q.e1 > q.e0) {
      prefetch_l2(scol + q.e0, static_cast<uint32_t>((q.e1 - q.e0) * 4));
      prefetch_l2(sval + q.e0, static_cast<uint32_t>((q.e1 - q.e0) * sizeof(T)));
    }
  };
  // indices of slots [j, j + UG) of the slice starting at e0 with slen slots (-1 past the end)
  auto load_idx = [&](int (&c)[UG], int64_t e0, int j, int slen) {
#pragma unroll
    for (int u = 0; u < UG; ++u) c[u] = j + u < slen ? ld_stream(scol + e0 + static_cast<int64_t>(j + u) * C + grp) : -1;
  };

  int i = next_valid(static_cast<int>(blockIdx.x) * kSpmmWarps + static_cast<int>(threadIdx.x >> 5));
  if (i >= total) return;
  int in = next_valid(i + wstride);
  Slice cur = load_slice(i), nxt = load_slice(in);
  prefetch_slice(cur);
  prefetch_slice(nxt);
  for (int b0 = 0; b0 < nb; b0 += NBG) { // passes over the warp's slices, NBG blocks each
    const int nbh = nb - b0 < NBG ? nb - b0 : NBG;
    const T* Xb = X + static_cast<int64_t>(b0) * bstride + sub * VEC;
    if (b0 > 0) { // start the walk again
      i = next_valid(static_cast<int>(blockIdx.x) * kSpmmWarps + static_cast<int>(threadIdx.x >> 5));
      in = next_valid(i + wstride);
      cur = load_slice(i);
      nxt = load_slice(in);
    }
    int slen = static_cast<int>((cur.e1 - cur.e0) / C);
    int j = 0;
    int c[UG];
    load_idx(c, cur.e0, 0, slen);
    T acc[NBG][VEC];
#pragma unroll
    for (int bb = 0; bb < NBG; ++bb)
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[bb][v] = T(0);
    while (true) {
      // gathers and values of the current group
      T x[UG][NBG][VEC];
      T a[UG];
#pragma unroll
      for (int u = 0; u < UG; ++u) {
        a[u] = c[u] >= 0 ? ld_stream(sval + cur.e0 + static_cast<int64_t>(j + u) * C + grp) : T(0);
#pragma unroll
        for (int bb = 0; bb < NBG; ++bb) {
          if (c[u] >= 0 && bb < nbh) load_row<T, VEC>(Xb + static_cast<int64_t>(bb) * bstride + c[u] * BS, x[u][bb]);
          else
#pragma unroll
            for (int v = 0; v < VEC; ++v) x[u][bb][v] = T(0);
        }
      }
      // indices of the next group: this slice's, else the next slice's first
      const bool last = j + UG >= slen;
      if (!last) load_idx(c, cur.e0, j + UG, slen);
      else load_idx(c, nxt.e0, 0, static_cast<int>((nxt.e1 - nxt.e0) / C));
#pragma unroll
      for (int u = 0; u < UG; ++u)
#pragma unroll
        for (int bb = 0; bb < NBG; ++bb)
#pragma unroll
          for (int v = 0; v < VEC; ++v) acc[bb][v] = fma(a[u], x[u][bb][v], acc[bb][v]);
      if (!last) {
        j += UG;
        continue;
      }
      // the slice is complete: write its rows
      if (cur.row >= 0) {
#pragma unroll
        for (int bb = 0; bb < NBG; ++bb) {
          if (bb >= nbh) break;
          const int64_t off = static_cast<int64_t>(b0 + bb) * bstride + static_cast<int64_t>(cur.row) * BS + sub * VEC;
          T y[VEC];
          if (beta != T(0)) {
            T xr[VEC];
            load_row<T, VEC>(X + off, xr);
#pragma unroll
            for (int v = 0; v < VEC; ++v) y[v] = fma(alpha, acc[bb][v], beta * xr[v]); // explicit: the same rounding as the CSR kernel
          }
          else {
#pragma unroll
            for (int v = 0; v < VEC; ++v) y[v] = alpha * acc[bb][v];
          }
          if (W) { // W may be Y itself: this lane reads its values before it writes them
#pragma unroll
            for (int v = 0; v < VEC; ++v) y[v] = fma(gamma, W[off + v], y[v]);
          }
          store_row<T, VEC>(Y + off, y);
        }
      }
#pragma unroll
      for (int bb = 0; bb < NBG; ++bb)
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc[bb][v] = T(0);
      if (in >= total) break;
      i = in;
      in = next_valid(i + wstride);
      cur = nxt;
      nxt = load_slice(in);
      if (b0 == 0) prefetch_slice(nxt);
      slen = static_cast<int>((cur.e1 - cur.e0) / C);
      j = 0;
    }
  }
}

} // namespace

struct trl_cuda_sell_op {
  int device = 0;
  int dtype = TRL_F64;
  int bs = 0;
  int C = 0;
  int64_t n = 0, nnz = 0;
  int64_t nslices = 0, nwin = 0;
  int spw = 0;           // slices per window
  int interleave = 0;    // take slices window-major (skewed row lengths)
  int long_rows = 0;     // 16 or more slots per slice on average
  int64_t stored = 0;    // entries including padding
  int longest = 0;       // longest row (entries)
  int32_t* perm = nullptr;
  int64_t* sptr = nullptr;
  int32_t* scol = nullptr;
  void* sval = nullptr;
};

extern "C" {

int trl_cuda_op_destroy(trl_cuda_handle h, trl_cuda_op op)
{
  TRL_CHECK_HANDLE(h);
  if (!op) return TRL_OK;
  int st = TRL_OK;
  for (void* p : {static_cast<void*>(op->perm), static_cast<void*>(op->sptr), static_cast<void*>(op->scol), op->sval})
    if (p) {
      const int s = trl_cuda_free(h, p);
      if (s && !st) st = s;
    }
  delete op;
  return st;
}

int trl_cuda_op_create(trl_cuda_handle h, const trl_csr* A, int bs, trl_cuda_op* out)
{
  TRL_CHECK_HANDLE(h);
  if (!out) return set_error(h, TRL_EINVAL, "null output");
  *out = nullptr;
  if (!A) return set_error(h, TRL_EINVAL, "null operator");
  if (!valid_dtype(A->value_dtype)) return set_error(h, TRL_ENOTSUP, "unsupported value dtype %d", A->value_dtype);
  if (!valid_bs(bs)) return set_error(h, TRL_ENOTSUP, "unsupported block size %d", bs);
  if (A->n < 0 || A->nnz < 0 || A->nnz >= (int64_t(1) << 31) || A->n >= (int64_t(1) << 31) - kSellWindow) return set_error(h, TRL_EINVAL, "bad CSR sizes");
  if (A->n > 0 && (!A->rowptr || (A->nnz > 0 && (!A->colind || !A->values)))) return set_error(h, TRL_EINVAL, "null CSR array");
  auto* op = new trl_cuda_sell_op;
  op->device = h->device;
  op->dtype = A->value_dtype;
  op->bs = bs;
  op->n = A->n;
  op->nnz = A->nnz;
  op->C = A->value_dtype == TRL_F64 ? slice_height_for<double>(bs) : slice_height_for<float>(bs);
  const int C = op->C;
  op->nslices = (A->n + C - 1) / C;
  op->nwin = (A->n + kSellWindow - 1) / kSellWindow;
  op->spw = kSellWindow / C;
  if (A->n == 0) {
    *out = op;
    return TRL_OK;
  }
  const size_t es = A->value_dtype == TRL_F64 ? 8 : 4;
  const int64_t nparts = (op->nslices + kScanItems - 1) / kScanItems;
  int st = TRL_OK;
  auto fail = [&](int s) {
    trl_cuda_op_destroy(h, op);
    return s;
  };
  void* p = nullptr;
  if ((st = trl_cuda_malloc(h, &p, sizeof(int32_t) * op->nwin * kSellWindow))) return fail(st);
  op->perm = static_cast<int32_t*>(p);
  if ((st = trl_cuda_malloc(h, &p, sizeof(int64_t) * (op->nslices + 1)))) return fail(st);
  op->sptr = static_cast<int64_t*>(p);
  // scratch: per-CTA scan totals and {total entries, longest row}
  int64_t* part = static_cast<int64_t*>(workspace(h, sizeof(int64_t) * (nparts + 4)));
  if (!part) return fail(TRL_ENOMEM);
  auto* stats = reinterpret_cast<unsigned long long*>(part + nparts);
  cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), h->stream);
  launch(k_sell_sort, static_cast<unsigned>((op->nwin + kBuildWarps - 1) / kBuildWarps), kBuildThreads, 0, h->stream, A->n, op->nwin, A->rowptr, op->perm);
  if ((st = after_launch(h, "sell sort"))) return fail(st);
  launch(k_sell_slices, static_cast<unsigned>(nparts), 256, 0, h->stream, op->nslices, C, A->rowptr, op->perm, op->sptr, part, stats);
  if ((st = after_launch(h, "sell slices"))) return fail(st);
  launch(k_sell_scan_parts, 1, 1024, 0, h->stream, nparts, part, op->sptr, stats);
  if ((st = after_launch(h, "sell scan"))) return fail(st);
  launch(k_sell_add_parts, static_cast<unsigned>((op->nslices + 255) / 256), 256, 0, h->stream, op->nslices, part, op->sptr);
  if ((st = after_launch(h, "sell scan"))) return fail(st);
  unsigned long long hs[2] = {0, 0};
  if ((st = trl_cuda_memcpy(h, hs, stats, sizeof hs, TRL_D2H))) return fail(st);
  op->stored = static_cast<int64_t>(hs[0]);
  op->longest = static_cast<int>(hs[1]);
  // skewed row lengths (a slice far longer than the mean): spread each window's first slices
  const double mean = static_cast<double>(op->stored) / (static_cast<double>(op->nslices) * C);
  op->interleave = op->longest > 4.0 * mean + 8.0 ? 1 : 0;
  op->long_rows = mean >= 16.0 ? 1 : 0;
  const int64_t alloc = op->stored > 0 ? op->stored : 1;
  if ((st = trl_cuda_malloc(h, &p, sizeof(int32_t) * alloc))) return fail(st);
  op->scol = static_cast<int32_t*>(p);
  if ((st = trl_cuda_malloc(h, &p, es * alloc))) return fail(st);
  op->sval = p;
  if (op->stored > 0) {
    const unsigned grid = grid_for(h, op->nslices, kBuildWarps, 8);
    if (A->value_dtype == TRL_F64)
      launch(k_sell_fill<double>, grid, kBuildThreads, 0, h->stream, op->nslices, C, A->rowptr, A->colind, static_cast<const double*>(A->values), op->perm, op->sptr, op->scol,
                                                                  static_cast<double*>(op->sval));
    else
      launch(k_sell_fill<float>, grid, kBuildThreads, 0, h->stream, op->nslices, C, A->rowptr, A->colind, static_cast<const float*>(A->values), op->perm, op->sptr, op->scol,
                                                                 static_cast<float*>(op->sval));
    if ((st = after_launch(h, "sell fill"))) return fail(st);
  }
  *out = op;
  return TRL_OK;
}

int trl_cuda_op_info(trl_cuda_op op, int64_t* stored_entries, int* slice_height, int* longest_row)
{
  if (!op) return TRL_EINVAL;
  if (stored_entries) *stored_entries = op->stored;
  if (slice_height) *slice_height = op->C;
  if (longest_row) *longest_row = op->longest;
  return TRL_OK;
}

int trl_cuda_op_spmm(trl_cuda_handle h, trl_cuda_op op, const void* X, void* Y, int nb, double alpha, double beta, double gamma, const void* W)
{
  TRL_CHECK_HANDLE(h);
  if (!op) return set_error(h, TRL_EINVAL, "null operator");
  if (op->device != h->device) return set_error(h, TRL_EINVAL, "operator prepared on device %d, handle on device %d", op->device, h->device);
  if (nb < 1) return set_error(h, TRL_EINVAL, "block count %d", nb);
  if (!X || !Y) return set_error(h, TRL_EINVAL, "null pointer");
  if (op->n == 0) return TRL_OK;
  const int bs = op->bs;
  const size_t es = op->dtype == TRL_F64 ? 8 : 4;
  const auto overlap = [&](const void* a, const void* b) {
    const auto pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = static_cast<uintptr_t>(nb) * op->n * bs * es;
    return pa < pb + len && pb < pa + len;
  };
  if (overlap(X, Y) || (W && overlap(W, X)) || (W && W != Y && overlap(W, Y)))
    return set_error(h, TRL_EINVAL, "SpMM input must overlap neither output nor third operand");
  if (((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y) | reinterpret_cast<uintptr_t>(W)) % (es * bs < 32 ? es * bs : 32)) != 0)
    return set_error(h, TRL_EINVAL, "block vectors must be aligned to min(32, bs*elem) bytes");
  // algorithmic bytes of the CSR operator it was prepared from (the padding and the row
  // permutation are not credited)
  ProfScope prof(h, PROF_SPMM, op->nnz * (es + 4.0) + 4.0 * (op->n + 1) + nb * (W ? 3.0 : 2.0) * op->n * bs * es, 2.0 * op->nnz * bs * nb);
  int st = TRL_OK;
  const int dtype = op->dtype;
  TRL_DISPATCH_DT(dtype, TRL_DISPATCH_BS(bs, {
    const auto run = [&](auto kernel, int minb) {
      static int resident[64]; // per device and instantiation of the kernel
      int& res = resident[h->device & 63];
      if (res == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res, kernel, kSpmmThreads, 0) != cudaSuccess || res < 1) res = minb;
        cudaGetLastError();
      }
      // one resident wave; every warp strides over the slices
      const unsigned grid = grid_for(h, op->nslices, kSpmmWarps, res);
      trl_detail::launch(kernel, grid, kSpmmThreads, 0, h->stream, static_cast<int>(op->nslices), static_cast<int>(op->nwin), op->spw, op->interleave, op->perm, op->sptr, op->scol, static_cast<const T*>(op->sval),
                                                   static_cast<const T*>(X), static_cast<T*>(Y), static_cast<T>(alpha), static_cast<T>(beta), static_cast<T>(gamma),
                                                   static_cast<const T*>(W), nb, op->n * BS);
    };
    if (nb > 1) run(k_spmm_sell<T, BS, kSellBlocksPerPass, false>, SellTune<T, BS, kSellBlocksPerPass, false>::MINB);
    else if (op->long_rows) run(k_spmm_sell<T, BS, 1, true>, SellTune<T, BS, 1, true>::MINB);
    else run(k_spmm_sell<T, BS, 1, false>, SellTune<T, BS, 1, false>::MINB);
    st = after_launch(h, "spmm (sliced ELL)");
  }));
  return st;
}

} // extern "C"
