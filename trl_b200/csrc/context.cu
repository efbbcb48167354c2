// Handle, memory and error plumbing of the C ABI (include/trl_cuda.h).
#include "common.cuh"

#include <cstdarg>
#include <cstdlib>
#include <new>

namespace trl_detail {

int set_error(trl_cuda_context* h, int status, const char* fmt, ...)
{
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    h->last_error = buf;
  }
  return status;
}

bool pdl_enabled()
{
  static const bool on = [] {
    const char* v = std::getenv("TRL_PDL");
    return !(v && v[0] == '0');
  }();
  return on;
}

int after_launch(trl_cuda_context* h, const char* what)
{
  ++h->launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return TRL_OK;
}

void* workspace(trl_cuda_context* h, size_t bytes)
{
  if (bytes <= h->ws_bytes) return h->ws;
  // Growing: the old buffer may still be read by queued kernels on this stream.
  if (h->ws) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_bytes = 0;
  }
  size_t want = bytes < (size_t(1) << 20) ? (size_t(1) << 20) : bytes + bytes / 4;
  if (cudaMalloc(&h->ws, want) != cudaSuccess) {
    cudaGetLastError();
    set_error(h, TRL_ENOMEM, "workspace allocation of %zu bytes failed", want);
    return nullptr;
  }
  h->ws_bytes = want;
  return h->ws;
}

void* workspace2(trl_cuda_context* h, size_t bytes)
{
  if (bytes <= h->ws2_bytes) return h->ws2;
  if (h->ws2) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->ws2);
    h->ws2 = nullptr;
    h->ws2_bytes = 0;
  }
  size_t want = bytes < 65536 ? 65536 : bytes + bytes / 4;
  if (cudaMalloc(&h->ws2, want) != cudaSuccess) {
    cudaGetLastError();
    set_error(h, TRL_ENOMEM, "workspace allocation of %zu bytes failed", want);
    return nullptr;
  }
  h->ws2_bytes = want;
  return h->ws2;
}

void* pinned(trl_cuda_context* h, size_t bytes)
{
  if (bytes <= h->pinned_bytes) return h->pinned;
  if (h->pinned) {
    cudaStreamSynchronize(h->stream);
    cudaFreeHost(h->pinned);
    h->pinned = nullptr;
    h->pinned_bytes = 0;
  }
  size_t want = bytes < 65536 ? 65536 : bytes;
  if (cudaMallocHost(&h->pinned, want) != cudaSuccess) {
    cudaGetLastError();
    set_error(h, TRL_ENOMEM, "pinned allocation of %zu bytes failed", want);
    return nullptr;
  }
  h->pinned_bytes = want;
  return h->pinned;
}

cudaEvent_t prof_event(trl_cuda_context* h)
{
  if (!h->prof_free.empty()) {
    cudaEvent_t e = h->prof_free.back();
    h->prof_free.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void prof_resolve(trl_cuda_context* h)
{
  for (auto& p : h->prof_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      auto& s = h->prof[p.cls];
      s.calls += 1;
      s.seconds += ms * 1e-3;
      s.bytes += p.bytes;
      s.flops += p.flops;
    }
    else {
      cudaGetLastError();
    }
    h->prof_free.push_back(p.a);
    h->prof_free.push_back(p.b);
  }
  h->prof_pending.clear();
}

} // namespace trl_detail

using namespace trl_detail;

static const char* kProfNames[TRL_PROF_CLASSES] = {"spmm", "block_dot", "block_update", "block_rotate", "bv_mult", "cholqr",
                                                    "bv_sub", "small_eigen", "copy", "sddmm", "block_ops", "reorth_pass2"};

extern "C" int trl_cuda_profile_enable(trl_cuda_handle h, int on)
{
  TRL_CHECK_HANDLE(h);
  if (on) {
    cudaStreamSynchronize(h->stream);
    prof_resolve(h);
    for (int i = 0; i < TRL_PROF_CLASSES; ++i) {
      h->prof[i] = trl_kernel_stats{};
      std::snprintf(h->prof[i].name, sizeof h->prof[i].name, "%s", kProfNames[i]);
    }
  }
  h->profiling = on != 0;
  return TRL_OK;
}

extern "C" int trl_cuda_profile_read(trl_cuda_handle h, trl_kernel_stats* out)
{
  TRL_CHECK_HANDLE(h);
  if (!out) return set_error(h, TRL_EINVAL, "null output");
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "stream synchronize: %s", cudaGetErrorString(e));
  prof_resolve(h);
  for (int i = 0; i < TRL_PROF_CLASSES; ++i) {
    out[i] = h->prof[i];
    std::snprintf(out[i].name, sizeof out[i].name, "%s", kProfNames[i]);
  }
  return TRL_OK;
}

extern "C" {

int trl_cuda_create(trl_cuda_handle* out, int device, void* stream)
{
  if (!out) return TRL_EINVAL;
  *out = nullptr;
  auto* h = new (std::nothrow) trl_cuda_context();
  if (!h) return TRL_ENOMEM;
  h->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return TRL_ECUDA;
  }
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  // NULL asks for a private stream; the legacy default stream is requested explicitly as
  // cudaStreamLegacy ((void*)1), the per-thread default stream as cudaStreamPerThread.
  if (stream) {
    h->stream = static_cast<cudaStream_t>(stream);
  }
  else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete h;
      return TRL_ECUDA;
    }
    h->owns_stream = true;
  }
  if (cudaMalloc(&h->d_status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    if (h->owns_stream) cudaStreamDestroy(h->stream);
    delete h;
    return TRL_ENOMEM;
  }
  if (cudaMallocHost(&h->pinned_status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(h->d_status);
    if (h->owns_stream) cudaStreamDestroy(h->stream);
    delete h;
    return TRL_ENOMEM;
  }
  cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream);
  *out = h;
  return TRL_OK;
}

int trl_cuda_destroy(trl_cuda_handle h)
{
  if (!h) return TRL_OK;
  cudaStreamSynchronize(h->stream);
  prof_resolve(h);
  for (cudaEvent_t e : h->prof_free) cudaEventDestroy(e);
  destroy_solver(h);
  if (h->pool) {
    cudaStreamSynchronize(h->stream);
    cudaMemPoolDestroy(h->pool); // its reserved memory goes back once every block is freed
  }
  if (h->ws) cudaFree(h->ws);
  if (h->ws2) cudaFree(h->ws2);
  if (h->d_small) cudaFree(h->d_small);
  if (h->pinned) cudaFreeHost(h->pinned);
  if (h->d_status) cudaFree(h->d_status);
  if (h->pinned_status) cudaFreeHost(h->pinned_status);
  if (h->owns_stream) cudaStreamDestroy(h->stream);
  delete h;
  return TRL_OK;
}

int trl_cuda_synchronize(trl_cuda_handle h)
{
  TRL_CHECK_HANDLE(h);
  int* st = h->pinned_status;
  cudaMemcpyAsync(st, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "stream synchronize: %s", cudaGetErrorString(e));
  if (!h->prof_pending.empty()) prof_resolve(h);
  const int flags = *st;
  if (flags & TRL_DEV_CHOLESKY) return set_error(h, TRL_ECHOLESKY, "Cholesky factorization failed in orthonormalize");
  if (flags & TRL_DEV_EIGEN) return set_error(h, TRL_EEIGEN, "Eigendecomposition failed");
  if (flags & TRL_DEV_TIMEOUT) return set_error(h, TRL_ETIMEOUT, "a bounded device wait timed out");
  return TRL_OK;
}

void* trl_cuda_stream(trl_cuda_handle h) { return h ? static_cast<void*>(h->stream) : nullptr; }

const char* trl_cuda_last_error(trl_cuda_handle h) { return h ? h->last_error.c_str() : "null handle"; }

uint64_t trl_cuda_launch_count(trl_cuda_handle h) { return h ? h->launches : 0; }

const char* trl_cuda_status_string(int s)
{
  switch (s) {
  case TRL_OK: return "ok";
  case TRL_EINVAL: return "invalid argument";
  case TRL_ENOMEM: return "out of device memory";
  case TRL_ECUDA: return "CUDA error";
  case TRL_ECHOLESKY: return "Cholesky factorization failed in orthonormalize";
  case TRL_EEIGEN: return "Eigendecomposition failed";
  case TRL_ETIMEOUT: return "device wait timed out";
  case TRL_ENOTSUP: return "unsupported block size or dtype";
  default: return "unknown status";
  }
}

// Buffers come from a memory pool owned by the handle whose release threshold keeps freed
// memory reserved, so the multi-GB bases of repeated solves are not returned to the driver
// and mapped again each time: measured on B200, cudaMalloc/cudaFree of a solve's buffers
// (4-6 GB in ~12 blocks) took 12 ms typically and up to 1.1 s of host time, during which the
// GPU idles.
int trl_cuda_malloc(trl_cuda_handle h, void** ptr, size_t bytes)
{
  TRL_CHECK_HANDLE(h);
  if (!ptr) return set_error(h, TRL_EINVAL, "null output pointer");
  *ptr = nullptr;
  if (bytes == 0) return TRL_OK;
  if (h->refuse_allocs > 0) {
    --h->refuse_allocs;
    return set_error(h, TRL_ENOMEM, "allocation of %zu bytes refused (injected failure)", bytes);
  }
  if (!h->pool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = h->device;
    if (cudaMemPoolCreate(&h->pool, &props) != cudaSuccess) {
      cudaGetLastError();
      h->pool = nullptr;
      return set_error(h, TRL_ECUDA, "memory pool creation failed");
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(h->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (cudaMallocFromPoolAsync(ptr, bytes, h->pool, h->stream) != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return set_error(h, TRL_ENOMEM, "allocation of %zu bytes failed", bytes);
  }
  // usable from any stream on return, as cudaMalloc memory is
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "allocation: %s", cudaGetErrorString(e));
  if (reinterpret_cast<uintptr_t>(*ptr) % 256 != 0) return set_error(h, TRL_ECUDA, "pool allocation not 256-byte aligned");
  return TRL_OK;
}

int trl_cuda_free(trl_cuda_handle h, void* ptr)
{
  TRL_CHECK_HANDLE(h);
  if (!ptr) return TRL_OK;
  cudaError_t e = cudaFreeAsync(ptr, h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "free: %s", cudaGetErrorString(e));
  return TRL_OK;
}

int trl_cuda_memcpy(trl_cuda_handle h, void* dst, const void* src, size_t bytes, int kind)
{
  TRL_CHECK_HANDLE(h);
  if (bytes == 0) return TRL_OK;
  if (!dst || !src) return set_error(h, TRL_EINVAL, "null pointer in memcpy");
  cudaMemcpyKind k;
  switch (kind) {
  case TRL_H2D: k = cudaMemcpyHostToDevice; break;
  case TRL_D2H: k = cudaMemcpyDeviceToHost; break;
  case TRL_D2D: k = cudaMemcpyDeviceToDevice; break;
  default: return set_error(h, TRL_EINVAL, "bad copy kind %d", kind);
  }
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, k, h->stream);
  if (e == cudaSuccess && kind == TRL_D2H) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "memcpy: %s", cudaGetErrorString(e));
  return TRL_OK;
}

int trl_cuda_memset_zero(trl_cuda_handle h, void* ptr, size_t bytes)
{
  TRL_CHECK_HANDLE(h);
  if (bytes == 0) return TRL_OK;
  if (!ptr) return set_error(h, TRL_EINVAL, "null pointer in memset");
  cudaError_t e = cudaMemsetAsync(ptr, 0, bytes, h->stream);
  if (e != cudaSuccess) return set_error(h, TRL_ECUDA, "memset: %s", cudaGetErrorString(e));
  return TRL_OK;
}

} // extern "C"

namespace {

// One thread waits on a shared-memory mbarrier that expects two arrivals and gets one: the
// phase never completes, the wait gives up after `polls` polls and records TRL_DEV_TIMEOUT.
__global__ void k_wait_never_completes(int* status, unsigned polls)
{
  ::trl_detail::pdl_enter();
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 2);
  mbar_arrive(&bar);
  mbar_wait(&bar, 0, status, polls);
}

} // namespace

extern "C" int trl_cuda_inject_alloc_failures(trl_cuda_handle h, int count)
{
  TRL_CHECK_HANDLE(h);
  if (count < 0) return set_error(h, TRL_EINVAL, "negative count");
  h->refuse_allocs = count;
  return TRL_OK;
}

extern "C" int trl_cuda_test_bounded_wait(trl_cuda_handle h, unsigned polls)
{
  TRL_CHECK_HANDLE(h);
  if (polls == 0 || polls > (1u << 24)) return set_error(h, TRL_EINVAL, "polls must be in [1, 2^24]");
  launch(k_wait_never_completes, 1, 32, 0, h->stream, h->d_status, polls);
  return after_launch(h, "bounded wait");
}
