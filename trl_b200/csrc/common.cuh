// Shared internals of libtrl_cuda.so (sm_100a). Not part of the public ABI.
#pragma once

#include "trl_cuda.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

// Device status word bits (sticky until trl_cuda_synchronize reads and clears them).
#define TRL_DEV_CHOLESKY 0x1
#define TRL_DEV_EIGEN 0x2
#define TRL_DEV_TIMEOUT 0x4

struct trl_cuda_context {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr; // trl_cuda_malloc's stream-ordered pool (created on first use)
  bool owns_stream = false;
  int* d_status = nullptr;  // device status word
  void* ws = nullptr;       // growable device workspace (per-call partial sums)
  void* ws2 = nullptr;      // growable device workspace (coefficients kept across calls of one operation)
  size_t ws2_bytes = 0;
  double* d_small = nullptr; // 1024 doubles of fixed scratch (Gram / factor blocks)
  size_t ws_bytes = 0;
  int* pinned_status = nullptr; // pinned host copy of d_status
  void* pinned = nullptr;   // small pinned host staging buffer
  size_t pinned_bytes = 0;
  void* solver = nullptr;   // cusolverDnHandle_t, created on first use
  void* syevd_work = nullptr;
  size_t syevd_work_bytes = 0;
  uint64_t launches = 0;
  int refuse_allocs = 0; // trl_cuda_inject_alloc_failures: allocations still to refuse
  std::string last_error;
  // per-kernel-class device timing (trl_cuda_profile_*)
  bool profiling = false;
  int prof_depth = 0;
  struct ProfPending {
    cudaEvent_t a, b;
    int cls;
    double bytes, flops;
  };
  std::vector<ProfPending> prof_pending;
  std::vector<cudaEvent_t> prof_free;
  trl_kernel_stats prof[TRL_PROF_CLASSES] = {};
};

namespace trl_detail {

int set_error(trl_cuda_context* h, int status, const char* fmt, ...);

// Ensures at least `bytes` of device workspace; returns nullptr and sets an error on failure.
void* workspace(trl_cuda_context* h, size_t bytes);
void* workspace2(trl_cuda_context* h, size_t bytes);
void* pinned(trl_cuda_context* h, size_t bytes);

inline bool valid_bs(int bs) { return bs == 1 || bs == 2 || bs == 4 || bs == 8 || bs == 16; }
inline bool valid_dtype(int dt) { return dt == TRL_F64 || dt == TRL_F32; }

// Checks cudaGetLastError after a launch and counts the launch.
int after_launch(trl_cuda_context* h, const char* what);

// 1024 doubles of per-handle device scratch (Gram / factor blocks); nullptr on failure.
void* small_scratch(trl_cuda_context* h);
// Releases the cuSOLVER handle and its workspace.
void destroy_solver(trl_cuda_context* h);

// Kernel classes of the profiler (index into trl_cuda_context::prof).
enum ProfClass { PROF_SPMM = 0, PROF_DOT, PROF_UPDATE, PROF_ROTATE, PROF_MULT, PROF_CHOLQR, PROF_SUB, PROF_SMALL_EIGEN, PROF_COPY, PROF_SDDMM, PROF_BLOCK_OPS, PROF_REORTH2 };

cudaEvent_t prof_event(trl_cuda_context* h);
// Folds completed timings into the per-class totals (after a stream synchronisation).
void prof_resolve(trl_cuda_context* h);

// Times one C-ABI call (outermost call only) with a pair of events on the handle's stream
// and credits it with the call's algorithmic bytes and flops.
class ProfScope {
public:
  ProfScope(trl_cuda_context* h, int cls, double bytes, double flops = 0.0)
      : h_(h)
      , cls_(cls)
      , bytes_(bytes)
      , flops_(flops)
  {
    if (!h_->profiling) return;
    counted_ = true;
    if (h_->prof_depth++ != 0) return;
    active_ = true;
    a_ = prof_event(h_);
    b_ = prof_event(h_);
    cudaEventRecord(a_, h_->stream);
  }
  ~ProfScope()
  {
    if (!counted_) return;
    --h_->prof_depth;
    if (!active_) return;
    cudaEventRecord(b_, h_->stream);
    h_->prof_pending.push_back({a_, b_, cls_, bytes_, flops_});
  }
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

private:
  trl_cuda_context* h_;
  int cls_;
  double bytes_, flops_;
  bool counted_ = false, active_ = false;
  cudaEvent_t a_{}, b_{};
};

// Grid sizing: a multiple of the SM count, capped by the work available.
inline unsigned grid_for(const trl_cuda_context* h, int64_t work_items, int items_per_cta, int ctas_per_sm)
{
  int64_t need = (work_items + items_per_cta - 1) / items_per_cta;
  int64_t cap = static_cast<int64_t>(h->num_sms) * ctas_per_sm;
  if (need < 1) need = 1;
  return static_cast<unsigned>(need < cap ? need : cap);
}

// Programmatic dependent launch. Every kernel of the library starts with pdl_enter(). A
// kernel launched by launch() below (programmatic stream serialization) may have its CTAs
// scheduled while the previous kernel of its stream is still finishing; they wait in
// griddepcontrol.wait until that kernel has completed and its memory operations are
// visible, before touching any global memory, so the ordering is that of a plain launch
// while the launch latency of a chain of short dependent kernels overlaps the tail of
// each predecessor. The trigger that follows lets this kernel's own successor be
// scheduled once all of its CTAs have passed the wait. For a kernel launched without the
// attribute both instructions return at once.
__device__ __forceinline__ void pdl_enter()
{
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// true unless the environment sets TRL_PDL=0 (read once per process)
bool pdl_enabled();

// kernel<<<grid, block, smem, stream>>>(args...) with programmatic stream serialization
// when pdl_enabled() and the stream is not the legacy default stream (whose implicit
// synchronisation with other streams is left as it is). Every kernel parameter is passed
// explicitly (no default arguments).
template <typename... P, typename... A>
cudaError_t launch(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, A&&... args)
{
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = (pdl_enabled() && stream != nullptr && stream != cudaStreamLegacy) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

} // namespace trl_detail

// FP64 tensor-core MMA, m8n8k4 (DMMA). Fragment layout (PTX ISA, mma.m8n8k4 .f64):
// with g = lane>>2 and t = lane&3: a = A[g][t], b = B[t][g], {d0,d1} = D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n" : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

template <typename T>
__device__ __forceinline__ double ld_widen(const T* p)
{
  return static_cast<double>(__ldg(p));
}

// ---- bulk-copy pipeline primitives (sm_90+ PTX; no cluster multicast anywhere) ------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes mbarrier initialisation visible to the asynchronous (bulk-copy) proxy
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Waits for the phase with the given parity to complete. Bounded: after `limit` polls it
// records TRL_DEV_TIMEOUT in the status word and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status, uint32_t limit = (1u << 24))
{
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  atomicOr(status, TRL_DEV_TIMEOUT);
  return false;
}

// 1-D bulk copy global -> shared, completing `bytes` transactions on `bar`. Both addresses
// 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// ---- vector loads shared by the SpMM kernels (spmm.cu, sell.cu) ---------------------------
namespace trl_detail {

template <typename T, int VEC>
struct VecT;
template <>
struct VecT<double, 1> {
  using type = double;
};
template <>
struct VecT<double, 2> {
  using type = double2;
};
template <>
struct VecT<float, 1> {
  using type = float;
};
template <>
struct VecT<float, 2> {
  using type = float2;
};
template <>
struct VecT<float, 4> {
  using type = float4;
};

template <typename T, int VEC>
__device__ __forceinline__ void load_vec(const T* p, T (&out)[VEC])
{
  using V = typename VecT<T, VEC>::type;
  const V v = __ldg(reinterpret_cast<const V*>(p));
  if constexpr (VEC == 1) {
    out[0] = reinterpret_cast<const T*>(&v)[0];
  }
  else {
#pragma unroll
    for (int i = 0; i < VEC; ++i) out[i] = reinterpret_cast<const T*>(&v)[i];
  }
}

template <typename T, int VEC>
__device__ __forceinline__ void store_vec(T* p, const T (&in)[VEC])
{
  using V = typename VecT<T, VEC>::type;
  V v;
#pragma unroll
  for (int i = 0; i < VEC; ++i) reinterpret_cast<T*>(&v)[i] = in[i];
  *reinterpret_cast<V*>(p) = v;
}

// The CSR stream is read once: load it without allocating in L1, which keeps L1 for the
// X rows that neighbouring rows gather again.
__device__ __forceinline__ int ld_stream(const int32_t* p)
{
  int v;
  asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p)
{
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p)
{
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

} // namespace trl_detail

#define TRL_CHECK_HANDLE(h)                                                                                                                                                                            \
  do {                                                                                                                                                                                                 \
    if (!(h)) return TRL_EINVAL;                                                                                                                                                                       \
  } while (0)

// Dispatch a block size to a compile-time constant BS.
#define TRL_DISPATCH_BS(bs, ...)                                                                                                                                                                       \
  switch (bs) {                                                                                                                                                                                        \
  case 1: {                                                                                                                                                                                            \
    constexpr int BS = 1;                                                                                                                                                                              \
    __VA_ARGS__;                                                                                                                                                                                       \
  } break;                                                                                                                                                                                             \
  case 2: {                                                                                                                                                                                            \
    constexpr int BS = 2;                                                                                                                                                                              \
    __VA_ARGS__;                                                                                                                                                                                       \
  } break;                                                                                                                                                                                             \
  case 4: {                                                                                                                                                                                            \
    constexpr int BS = 4;                                                                                                                                                                              \
    __VA_ARGS__;                                                                                                                                                                                       \
  } break;                                                                                                                                                                                             \
  case 8: {                                                                                                                                                                                            \
    constexpr int BS = 8;                                                                                                                                                                              \
    __VA_ARGS__;                                                                                                                                                                                       \
  } break;                                                                                                                                                                                             \
  case 16: {                                                                                                                                                                                           \
    constexpr int BS = 16;                                                                                                                                                                             \
    __VA_ARGS__;                                                                                                                                                                                       \
  } break;                                                                                                                                                                                             \
  default: return trl_detail::set_error(h, TRL_ENOTSUP, "unsupported block size %d", bs);                                                                                                             \
  }

#define TRL_DISPATCH_DT(dt, ...)                                                                                                                                                                       \
  if ((dt) == TRL_F64) {                                                                                                                                                                               \
    using T = double;                                                                                                                                                                                  \
    __VA_ARGS__;                                                                                                                                                                                       \
  }                                                                                                                                                                                                    \
  else if ((dt) == TRL_F32) {                                                                                                                                                                          \
    using T = float;                                                                                                                                                                                   \
    __VA_ARGS__;                                                                                                                                                                                       \
  }                                                                                                                                                                                                    \
  else                                                                                                                                                                                                 \
    return trl_detail::set_error(h, TRL_ENOTSUP, "unsupported dtype %d", dt);
