// Host-logic test of trl::cuda::Context's rotation batching, linked against a fake C ABI
// that records calls instead of launching kernels (no GPU needed). Prints one line per ABI
// call; tests/test_host_logic.py checks the sequences.
#include <trl/impl/cuda/context.hh>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

static std::vector<std::string> g_log;

extern "C" {
struct trl_cuda_context {
  int dummy;
};
static trl_cuda_context g_ctx;
int trl_cuda_create(trl_cuda_handle* h, int, void*)
{
  *h = &g_ctx;
  return TRL_OK;
}
int trl_cuda_destroy(trl_cuda_handle) { return TRL_OK; }
int trl_cuda_synchronize(trl_cuda_handle) { return TRL_OK; }
const char* trl_cuda_last_error(trl_cuda_handle) { return ""; }
const char* trl_cuda_status_string(int) { return "fake"; }
int trl_cuda_malloc(trl_cuda_handle, void** p, size_t bytes)
{
  *p = std::malloc(bytes ? bytes : 1);
  return TRL_OK;
}
int trl_cuda_free(trl_cuda_handle, void* p)
{
  std::free(p);
  return TRL_OK;
}
int trl_cuda_bv_zero(trl_cuda_handle, int, void* X, int64_t, int)
{
  g_log.push_back("zero " + std::to_string(reinterpret_cast<uintptr_t>(X)));
  return TRL_OK;
}
int trl_cuda_bv_mult(trl_cuda_handle, int, int mode, const void* X, const double* W, void* Y, int64_t, int)
{
  g_log.push_back("mult " + std::to_string(mode) + " " + std::to_string(reinterpret_cast<uintptr_t>(X)) + " " + std::to_string(reinterpret_cast<uintptr_t>(W)) + " " +
                  std::to_string(reinterpret_cast<uintptr_t>(Y)));
  return TRL_OK;
}
int trl_cuda_block_rotate(trl_cuda_handle, int, const void* V, int m, const double* Y, int ldy, int k, void* W, int64_t, int)
{
  g_log.push_back("rotate " + std::to_string(reinterpret_cast<uintptr_t>(V)) + " m=" + std::to_string(m) + " " + std::to_string(reinterpret_cast<uintptr_t>(Y)) +
                  " ldy=" + std::to_string(ldy) + " k=" + std::to_string(k) + " " + std::to_string(reinterpret_cast<uintptr_t>(W)));
  return TRL_OK;
}
}

int main()
{
  trl::cuda::Context ctx(0, nullptr);
  const int bs = 4;
  const std::int64_t n = 10;
  const std::ptrdiff_t blk = n * bs; // elements per block
  std::vector<double> V(20 * blk), W(20 * blk), Y(30 * 30 * bs * bs);
  auto Vb = [&](int i) { return V.data() + i * blk; };
  auto Wb = [&](int j) { return W.data() + j * blk; };
  auto Yb = [&](int i, int j, int ldy) { return Y.data() + (i * ldy + j) * bs * bs; };

  // 1) the thick-restart pattern (lanczos.hh:105-114): k=3, m=6, ldy=8 -> one rotation
  for (int j = 0; j < 3; ++j) {
    ctx.record_zero(TRL_F64, bs, n, Wb(j));
    for (int i = 0; i < 6; ++i) ctx.record_mult_add(TRL_F64, bs, n, Vb(i), Yb(i, j, 8), Wb(j));
  }
  ctx.flush();
  std::printf("case1 %zu %s\n", g_log.size(), g_log.empty() ? "" : g_log.back().c_str());
  std::printf("expect1 rotate %lu m=6 %lu ldy=8 k=3 %lu\n", (unsigned long)reinterpret_cast<uintptr_t>(V.data()), (unsigned long)reinterpret_cast<uintptr_t>(Y.data()),
              (unsigned long)reinterpret_cast<uintptr_t>(W.data()));
  g_log.clear();

  // 2) a gap in the basis blocks -> replay every call in order
  ctx.record_zero(TRL_F64, bs, n, Wb(0));
  ctx.record_mult_add(TRL_F64, bs, n, Vb(0), Yb(0, 0, 8), Wb(0));
  ctx.record_mult_add(TRL_F64, bs, n, Vb(2), Yb(1, 0, 8), Wb(0));
  ctx.flush();
  std::printf("case2 %zu %s | %s | %s\n", g_log.size(), g_log[0].substr(0, 4).c_str(), g_log[1].substr(0, 6).c_str(), g_log[2].substr(0, 6).c_str());
  g_log.clear();

  // 3) accumulation without a leading zero (mult_add onto existing data) -> replay
  ctx.record_mult_add(TRL_F64, bs, n, Vb(0), Yb(0, 0, 8), Wb(0));
  ctx.flush();
  std::printf("case3 %zu %s\n", g_log.size(), g_log[0].substr(0, 6).c_str());
  g_log.clear();

  // 4) output overlapping the input -> replay
  ctx.record_zero(TRL_F64, bs, n, Vb(1));
  ctx.record_mult_add(TRL_F64, bs, n, Vb(0), Yb(0, 0, 8), Vb(1));
  ctx.record_mult_add(TRL_F64, bs, n, Vb(1), Yb(1, 0, 8), Vb(1));
  ctx.flush();
  std::printf("case4 %zu\n", g_log.size());
  g_log.clear();

  // 5) a single input block (m = 1), k = 2 -> rotation with ldy >= k
  for (int j = 0; j < 2; ++j) {
    ctx.record_zero(TRL_F64, bs, n, Wb(j));
    ctx.record_mult_add(TRL_F64, bs, n, Vb(0), Yb(0, j, 5), Wb(j));
  }
  ctx.flush();
  std::printf("case5 %zu %s\n", g_log.size(), g_log.back().substr(0, 6).c_str());
  g_log.clear();

  // 6) a different block size in the middle flushes the first group on its own
  ctx.record_zero(TRL_F64, bs, n, Wb(0));
  ctx.record_mult_add(TRL_F64, bs, n, Vb(0), Yb(0, 0, 8), Wb(0));
  ctx.record_zero(TRL_F64, 8, n, Wb(5));
  ctx.flush();
  std::printf("case6 %zu %s %s\n", g_log.size(), g_log[0].substr(0, 6).c_str(), g_log[1].substr(0, 4).c_str());
  g_log.clear();

  // 7) batching disabled -> eager calls
  ctx.set_batching(false);
  ctx.record_zero(TRL_F64, bs, n, Wb(0));
  std::printf("case7 %zu\n", g_log.size());
  std::printf("fused %lu\n", (unsigned long)ctx.fused_rotations());
  return 0;
}
