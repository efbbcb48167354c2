// Host-logic test of trl::cuda::Context's rotation batching, three-term fusion and deferred
// writes, linked against a fake C ABI
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
int trl_cuda_bv_sub(trl_cuda_handle, int, void* X, const void* Y, int64_t, int)
{
  g_log.push_back("sub " + std::to_string(reinterpret_cast<uintptr_t>(X)) + " " + std::to_string(reinterpret_cast<uintptr_t>(Y)));
  return TRL_OK;
}
int trl_cuda_block_dot(trl_cuda_handle, int, const void* V, int nblk, const void* W, int64_t, int, double* C)
{
  g_log.push_back("dot " + std::to_string(reinterpret_cast<uintptr_t>(V)) + " " + std::to_string(nblk) + " " + std::to_string(reinterpret_cast<uintptr_t>(W)) + " " +
                  std::to_string(reinterpret_cast<uintptr_t>(C)));
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

  // 8) the driver's step i = 3 (lanczos.hh:243-262), then the projection: the calls run in
  //    order with each product/subtract pair as one kernel; W0 = V_3 T_33 is deferred
  auto u = [](const void* p) { return (unsigned long)reinterpret_cast<uintptr_t>(p); };
  const std::size_t blkb = sizeof(double) * blk, cb = sizeof(double) * bs * bs;
  std::vector<double> T(6 * 6 * bs * bs), B(2 * bs * bs);
  auto Tb = [&](int i, int j) { return T.data() + (i * 6 + j) * bs * bs; };
  double* beta = B.data();
  auto step = [&](int i) {
    ctx.record_mult(TRL_F64, bs, n, Vb(i - 1), beta, Wb(0), true);
    ctx.record_sub(TRL_F64, bs, n, Vb(i + 1), Wb(0));
    ctx.record_dot(TRL_F64, bs, n, Vb(i), Vb(i + 1), Tb(i, i));
    ctx.record_mult(TRL_F64, bs, n, Vb(i), Tb(i, i), Wb(0), false);
    ctx.record_sub(TRL_F64, bs, n, Vb(i + 1), Wb(0));
  };
  auto project = [&](int count, int w) { ctx.prepare({{Vb(0), blkb * count, false}, {Vb(w), blkb, false}, {Vb(w), blkb, true}}); };
  step(3);
  std::printf("case8a %zu\n", g_log.size()); // nothing issued yet
  project(4, 4);
  std::printf("case8 %zu %s | %s | %s\n", g_log.size(), g_log[0].c_str(), g_log[1].c_str(), g_log[2].c_str());
  std::printf("expect8 3 mult 4 %lu %lu %lu | dot %lu 1 %lu %lu | mult 3 %lu %lu %lu\n", u(Vb(2)), u(beta), u(Vb(4)), u(Vb(3)), u(Vb(4)), u(Tb(3, 3)), u(Vb(3)),
              u(Tb(3, 3)), u(Vb(4)));
  g_log.clear();
  // orthonormalize(V_4, beta), T(4,3) = beta, apply(V_4, V_5): none touches W0, V_3 or T_33;
  // the next step overwrites W0 first, so the deferred product is never written
  ctx.prepare({{Vb(4), blkb, false}, {Vb(4), blkb, true}, {beta, cb, true}});
  ctx.prepare({{beta, cb, false}, {Tb(4, 3), cb, true}});
  ctx.prepare({{Vb(4), blkb, false}, {Vb(5), blkb, true}});
  step(4);
  project(5, 5);
  std::printf("case8b %zu %lu %lu\n", g_log.size(), (unsigned long)ctx.deferred_writes(), (unsigned long)ctx.fused_pairs());
  g_log.clear();

  // 9) a later read of W0 writes the deferred product first (W0 = V_4 T_44)
  ctx.prepare({{Wb(0), blkb, false}});
  std::printf("case9 %zu %s\n", g_log.size(), g_log.empty() ? "" : g_log[0].c_str());
  std::printf("expect9 mult 0 %lu %lu %lu\n", u(Vb(4)), u(Tb(4, 4)), u(Wb(0)));
  g_log.clear();

  // 10) overwriting T_ii (an input of the deferred product) writes it first, too
  step(3);
  project(4, 4);
  g_log.clear();
  ctx.prepare({{Tb(3, 3), cb, true}});
  std::printf("case10 %zu %s\n", g_log.size(), g_log.empty() ? "" : g_log[0].substr(0, 6).c_str());
  g_log.clear();
  ctx.flush();
  std::printf("case10b %zu\n", g_log.size());

  // 11) the restart step (lanczos.hh:167-183): dot first, then the V_k and V_{k-1} products;
  //     flush() at the end writes the deferred W0 = V_4 T(5,4)^T
  ctx.record_dot(TRL_F64, bs, n, Vb(5), Vb(6), Tb(5, 5));
  ctx.record_mult(TRL_F64, bs, n, Vb(5), Tb(5, 5), Wb(0), false);
  ctx.record_sub(TRL_F64, bs, n, Vb(6), Wb(0));
  ctx.record_mult(TRL_F64, bs, n, Vb(4), Tb(5, 4), Wb(0), true);
  ctx.record_sub(TRL_F64, bs, n, Vb(6), Wb(0));
  ctx.flush();
  std::string seq;
  for (const auto& e : g_log) seq += e.substr(0, e.find(' ', e.find(' ') + 1)) + ",";
  std::printf("case11 %zu %s\n", g_log.size(), seq.c_str());
  g_log.clear();

  // 12) the reference's ModifiedGS after the step: its dot joins the record, and its
  //     subtract_product (an unrecorded operation) issues everything in order
  step(3);
  ctx.record_dot(TRL_F64, bs, n, Vb(0), Vb(4), B.data() + bs * bs);
  ctx.prepare({{Vb(0), blkb, false}, {B.data() + bs * bs, cb, false}, {Vb(4), blkb, false}, {Vb(4), blkb, true}});
  seq.clear();
  for (const auto& e : g_log) seq += e.substr(0, e.find(' ', e.find(' ') + 1)) + ",";
  std::printf("case12 %zu %s\n", g_log.size(), seq.c_str());
  g_log.clear();
  ctx.flush();
  g_log.clear();

  // 7) batching disabled -> eager calls
  ctx.set_batching(false);
  ctx.record_zero(TRL_F64, bs, n, Wb(0));
  std::printf("case7 %zu\n", g_log.size());
  g_log.clear();
  step(3);
  std::printf("case7b %zu\n", g_log.size());
  std::printf("fused %lu\n", (unsigned long)ctx.fused_rotations());
  return 0;
}
