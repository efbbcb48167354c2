// C entry points (include/trl_solver.h) that run trl's BlockLanczos driver, unchanged, on
// the CUDA backend. This translation unit is compiled against the reference's own headers
// (include/trl/eigensolvers/lanczos.hh, params.hh, reorthogonalization.hh, concepts.hh)
// and the backend headers in include/trl/impl/cuda/.
#include <trl/concepts.hh>
#include <trl/eigensolvers/lanczos.hh>
#include <trl/eigensolvers/params.hh>
#include <trl/eigensolvers/reorthogonalization.hh>

#include <trl/impl/cuda/csrevp.hh>
#include <trl/impl/cuda/reorthogonalization.hh>

#include "trl_solver.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <random>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

using trl::cuda::Context;
using trl::cuda::DeviceBuffer;
using trl::cuda::DeviceCSR;

static_assert(trl::Eigenproblem<trl::cuda::CSREVP<double, 8>>);
static_assert(trl::Eigenproblem<trl::cuda::CSREVP<float, 8>>);
static_assert(trl::ReorthogonalizationStrategy<trl::cuda::BlockCGS2, trl::cuda::CSREVP<double, 4>, trl::cuda::BlockMultivector<double, 4>>);

class EventTimer {
public:
  explicit EventTimer(cudaStream_t s)
      : s_(s)
  {
    cudaEventCreate(&a_);
    cudaEventCreate(&b_);
  }
  ~EventTimer()
  {
    cudaEventDestroy(a_);
    cudaEventDestroy(b_);
  }
  void start() { cudaEventRecord(a_, s_); }
  double stop()
  {
    cudaEventRecord(b_, s_);
    cudaEventSynchronize(b_);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a_, b_);
    return ms * 1e-3;
  }

private:
  cudaStream_t s_;
  cudaEvent_t a_{}, b_{};
};

struct PhaseOut {
  bool converged = false;
  unsigned restarts = 0;
  unsigned applies = 0;
  std::vector<double> evals; // all Ritz values of the last projected problem, |theta| descending
};

/// Runs BlockLanczos<CSREVP<Storage,bs>, Reorth> from the device block X0 and writes the
/// first `kx` blocks of Ritz vectors (block layout, Storage) to ritz_out.
template <class Storage, unsigned bs, class Reorth>
PhaseOut run_phase(const std::shared_ptr<Context>& ctx, const trl_csr* A, const trl_solve_params& p, unsigned max_restarts, double tol, const Storage* X0, unsigned kx,
                   Storage* ritz_out)
{
  using EVP = trl::cuda::CSREVP<Storage, bs>;
  auto Adev = DeviceCSR<Storage>::wrap(A->n, A->nnz, A->rowptr, A->colind, static_cast<const Storage*>(A->values));
  auto evp = std::make_shared<EVP>(ctx, std::move(Adev), p.alpha, p.beta);
  evp->set_cholqr_passes(p.cholqr_passes);
  trl::EigensolverParams ep{.nev = p.nev, .ncv = p.ncv, .max_restarts = max_restarts, .tolerance = tol};
  trl::BlockLanczos<EVP, Reorth> lanczos(evp, ep);
  auto V0 = lanczos.initial_block();
  const auto h = ctx->handle();
  ctx->flush(); // direct ABI calls follow
  ctx->check(trl_cuda_memcpy(h, V0.data_, X0, sizeof(Storage) * static_cast<std::size_t>(A->n) * bs, TRL_D2D), "initial block");

  const auto res = lanczos.solve();
  ctx->flush();

  PhaseOut out;
  out.converged = res.converged;
  out.restarts = res.iterations;
  out.applies = res.n_op_apply;
  out.evals = evp->get_current_eigenvalues();
  if (ritz_out && kx > 0) {
    auto& V = lanczos.get_basis();
    const int m = static_cast<int>(p.ncv / bs);
    const auto n = static_cast<std::int64_t>(A->n);
    if (res.converged) {
      // x_c = sum_i V_i Y(i, c): the basis and the eigenvectors of the last projected problem
      const auto& Y = evp->get_current_eigenvectors();
      ctx->check(trl_cuda_block_rotate(h, trl::cuda::dtype_of<Storage>::value, V.data(), m, Y.data(), static_cast<int>(Y.block_cols()), static_cast<int>(kx), ritz_out, n, bs),
                 "ritz vectors");
    }
    else {
      // the solve ran out of restarts after a restart: blocks 0..k-1 of V already hold the
      // kept Ritz vectors of the last projected problem (lanczos.hh:105-118)
      ctx->check(trl_cuda_memcpy(h, ritz_out, V.data(), sizeof(Storage) * static_cast<std::size_t>(n) * bs * kx, TRL_D2D), "ritz vectors");
    }
  }
  ctx->sync();
  return out;
}

template <class Storage, unsigned bs>
PhaseOut run_phase_r(const std::shared_ptr<Context>& ctx, const trl_csr* A, const trl_solve_params& p, unsigned max_restarts, double tol, const Storage* X0, unsigned kx,
                     Storage* ritz_out)
{
  switch (p.reorth) {
  case TRL_REORTH_MGS: return run_phase<Storage, bs, trl::ModifiedGS>(ctx, A, p, max_restarts, tol, X0, kx, ritz_out);
  case TRL_REORTH_CGS2: return run_phase<Storage, bs, trl::cuda::BlockCGS2>(ctx, A, p, max_restarts, tol, X0, kx, ritz_out);
  case TRL_REORTH_CGS1: return run_phase<Storage, bs, trl::cuda::BlockCGS1>(ctx, A, p, max_restarts, tol, X0, kx, ritz_out);
  default: return run_phase<Storage, bs, trl::cuda::BlockCGSIfNeeded>(ctx, A, p, max_restarts, tol, X0, kx, ritz_out);
  }
}

template <unsigned bs>
int solve_device(const std::shared_ptr<Context>& ctx, const trl_solve_params& p, const trl_csr* A64, const trl_csr* A32, const double* X0, double* evals_host,
                 double* evecs_dev, double* resid_host, trl_solve_info* info)
{
  const auto h = ctx->handle();
  const std::int64_t n = A64->n;
  const unsigned kx = (p.nev + bs - 1) / bs; // blocks of Ritz vectors to form
  const unsigned kr = p.nev / bs + 1;        // blocks the thick restart keeps (lanczos.hh:97)
  cudaStream_t stream = static_cast<cudaStream_t>(trl_cuda_stream(h));
  const auto launches0 = trl_cuda_launch_count(h);

  EventTimer total(stream), phase(stream);
  total.start();
  DeviceBuffer X64(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs * std::max(kx, kr));
  PhaseOut out;
  double t32 = 0.0;

  if (p.mode == TRL_MODE_FP64) {
    out = run_phase_r<double, bs>(ctx, A64, p, p.max_restarts, p.tol, X0, p.want_vectors ? kx : 0, static_cast<double*>(X64.get()));
  }
  else {
    if (!A32) throw std::invalid_argument("FP32 and mixed modes need the FP32 copy of the operator");
    DeviceBuffer X32(ctx, sizeof(float) * static_cast<std::size_t>(n) * bs * std::max(kx, kr));
    DeviceBuffer X0f(ctx, sizeof(float) * static_cast<std::size_t>(n) * bs);
    ctx->check(trl_cuda_convert(h, TRL_F32, X0f.get(), TRL_F64, X0, n * bs), "initial block");
    if (p.mode == TRL_MODE_FP32) {
      out = run_phase_r<float, bs>(ctx, A32, p, p.max_restarts, p.tol, static_cast<const float*>(X0f.get()), kx, static_cast<float*>(X32.get()));
      ctx->check(trl_cuda_convert(h, TRL_F64, X64.get(), TRL_F32, X32.get(), n * bs * kx), "widen");
    }
    else {
      phase.start();
      PhaseOut o32 = run_phase_r<float, bs>(ctx, A32, p, p.max_restarts, p.fp32_tol, static_cast<const float*>(X0f.get()), kr, static_cast<float*>(X32.get()));
      t32 = phase.stop();
      info->restarts_fp32 = o32.restarts;
      info->n_op_apply_fp32 = o32.applies;
      // FP64 refinement: widen the kept FP32 Ritz vectors and start the FP64 solve from a
      // seeded random combination of them (the start block then carries every wanted
      // direction to FP32 accuracy).
      ctx->check(trl_cuda_convert(h, TRL_F64, X64.get(), TRL_F32, X32.get(), n * bs * kr), "widen");
      std::vector<double> G(static_cast<std::size_t>(kr) * bs * bs);
      std::mt19937 rng(p.seed);
      std::normal_distribution<double> dist;
      for (auto& g : G) g = dist(rng);
      DeviceBuffer Gd(ctx, sizeof(double) * G.size());
      ctx->check(trl_cuda_memcpy(h, Gd.get(), G.data(), sizeof(double) * G.size(), TRL_H2D), "refine coefficients");
      DeviceBuffer V0(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs);
      ctx->check(trl_cuda_block_rotate(h, TRL_F64, X64.get(), static_cast<int>(kr), static_cast<const double*>(Gd.get()), 1, 1, V0.get(), n, bs), "refine start");
      ctx->check(trl_cuda_synchronize(h), "refine start");
      out = run_phase_r<double, bs>(ctx, A64, p, p.refine_max_restarts, p.tol, static_cast<const double*>(V0.get()), p.want_vectors ? kx : 0,
                                    static_cast<double*>(X64.get()));
    }
  }
  info->converged = out.converged ? 1 : 0;
  info->restarts = out.restarts;
  info->n_op_apply = out.applies;
  info->seconds_fp32 = t32;
  for (unsigned c = 0; c < p.nev; ++c) evals_host[c] = c < out.evals.size() ? out.evals[c] : 0.0;

  // ---- Ritz vectors and true residuals, FP64 ----
  info->max_rel_residual = info->max_theta_residual = 0.0;
  if (p.want_vectors) {
    phase.start();
    double norm1 = 0.0;
    ctx->check(trl_cuda_csr_norm1(h, A64, p.alpha, p.beta, &norm1), "norm");
    info->op_norm1 = norm1;
    DeviceBuffer R(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs);
    DeviceBuffer D(ctx, sizeof(double) * bs * bs);
    DeviceBuffer G(ctx, sizeof(double) * bs * bs * 2);
    std::vector<double> gh(2 * bs * bs);
    for (unsigned j = 0; j < kx; ++j) {
      const double* Xj = static_cast<const double*>(X64.get()) + static_cast<std::size_t>(j) * n * bs;
      ctx->check(trl_cuda_spmm(h, A64, TRL_F64, Xj, R.get(), bs, p.alpha, p.beta), "residual");
      double diag[16] = {0};
      for (unsigned c = 0; c < bs; ++c) diag[c] = (j * bs + c < p.nev) ? evals_host[j * bs + c] : 0.0;
      ctx->check(trl_cuda_mb_zero(h, static_cast<double*>(D.get()), bs), "residual");
      ctx->check(trl_cuda_mb_set_diagonal(h, static_cast<double*>(D.get()), diag, bs), "residual");
      ctx->check(trl_cuda_bv_mult(h, TRL_F64, TRL_SUBTRACT, Xj, static_cast<const double*>(D.get()), R.get(), n, bs), "residual");
      ctx->check(trl_cuda_block_dot(h, TRL_F64, R.get(), 1, R.get(), n, bs, static_cast<double*>(G.get())), "residual");
      ctx->check(trl_cuda_block_dot(h, TRL_F64, Xj, 1, Xj, n, bs, static_cast<double*>(G.get()) + bs * bs), "residual");
      ctx->check(trl_cuda_memcpy(h, gh.data(), G.get(), sizeof(double) * 2 * bs * bs, TRL_D2H), "residual");
      for (unsigned c = 0; c < bs && j * bs + c < p.nev; ++c) {
        const double rn = std::sqrt(std::max(0.0, gh[c * bs + c]));
        const double xn = std::sqrt(std::max(0.0, gh[bs * bs + c * bs + c]));
        const double r_rel = rn / std::max(xn, 1e-300);
        const double rel = r_rel / std::max(norm1, 1e-300);
        const double theta_rel = r_rel / std::max(std::abs(evals_host[j * bs + c]), 1e-300);
        if (resid_host) resid_host[j * bs + c] = rel;
        info->max_rel_residual = std::max(info->max_rel_residual, rel);
        info->max_theta_residual = std::max(info->max_theta_residual, theta_rel);
      }
    }
    if (evecs_dev) ctx->check(trl_cuda_unblock(h, static_cast<const double*>(X64.get()), n, bs, static_cast<int>(p.nev), evecs_dev), "ritz vectors");
    ctx->sync();
    info->seconds_vectors = phase.stop();
  }
  info->seconds = total.stop();
  info->kernel_launches = trl_cuda_launch_count(h) - launches0;
  return TRL_OK;
}

int dispatch(const std::shared_ptr<Context>& ctx, const trl_solve_params& p, const trl_csr* A64, const trl_csr* A32, const double* X0, double* evals_host, double* evecs_dev,
             double* resid_host, trl_solve_info* info)
{
  switch (p.bs) {
  case 1: return solve_device<1>(ctx, p, A64, A32, X0, evals_host, evecs_dev, resid_host, info);
  case 2: return solve_device<2>(ctx, p, A64, A32, X0, evals_host, evecs_dev, resid_host, info);
  case 4: return solve_device<4>(ctx, p, A64, A32, X0, evals_host, evecs_dev, resid_host, info);
  case 8: return solve_device<8>(ctx, p, A64, A32, X0, evals_host, evecs_dev, resid_host, info);
  case 16: return solve_device<16>(ctx, p, A64, A32, X0, evals_host, evecs_dev, resid_host, info);
  default: throw std::invalid_argument("unsupported block size " + std::to_string(p.bs));
  }
}

int fail(const std::exception& e, int status)
{
  g_err = e.what();
  return status;
}

void validate(const trl_solve_params* p)
{
  if (!p) throw std::invalid_argument("null params");
  if (p->mode < TRL_MODE_FP64 || p->mode > TRL_MODE_MIXED) throw std::invalid_argument("bad mode");
  if (p->ncv % p->bs != 0) throw std::invalid_argument("ncv must be a multiple of the block size");
  if (p->cholqr_passes < 1 || p->cholqr_passes > 4) throw std::invalid_argument("cholqr_passes must be in [1, 4]");
  if (p->reorth < TRL_REORTH_MGS || p->reorth > TRL_REORTH_CGS1) throw std::invalid_argument("bad reorth strategy");
}

} // namespace

extern "C" {

void trl_solve_params_default(trl_solve_params* p)
{
  if (!p) return;
  *p = trl_solve_params{};
  p->bs = 8;
  p->mode = TRL_MODE_FP64;
  p->nev = 16;
  p->ncv = 64;
  p->max_restarts = 1000;
  p->tol = 1e-8;
  p->alpha = 1.0;
  p->beta = 0.0;
  p->reorth = TRL_REORTH_CGS_IFNEEDED;
  p->cholqr_passes = 2;
  p->fp32_tol = 1e-5;
  p->refine_max_restarts = 1000;
  p->want_vectors = 1;
  p->batching = 1;
  p->seed = 42;
}

const char* trl_solver_last_error(void) { return g_err.c_str(); }

int trl_solve_csr_device(trl_cuda_handle h, const trl_solve_params* p, const trl_csr* A64, const trl_csr* A32, const double* X0, double* evals_host, double* evecs_dev,
                         double* resid_host, trl_solve_info* info)
{
  try {
    validate(p);
    if (!h || !A64 || !X0 || !evals_host || !info) throw std::invalid_argument("null argument");
    *info = trl_solve_info{};
    // The solver's objects run on the caller's handle (its stream, workspace and profiler).
    auto ctx = Context::borrow(h);
    ctx->set_batching(p->batching != 0);
    return dispatch(ctx, *p, A64, A32, X0, evals_host, evecs_dev, resid_host, info);
  }
  catch (const std::invalid_argument& e) {
    return fail(e, TRL_EINVAL);
  }
  catch (const std::exception& e) {
    const std::string w = e.what();
    return fail(e, w.find("Cholesky") != std::string::npos ? TRL_ECHOLESKY : (w.find("Eigendecomposition") != std::string::npos ? TRL_EEIGEN : TRL_ECUDA));
  }
}

int trl_solve_csr_host(const trl_solve_params* p, int device, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind, const double* values, const double* X0,
                       double* evals, double* evecs, double* resid, trl_solve_info* info)
{
  try {
    validate(p);
    if (!rowptr || !X0 || !evals || !info || (nnz > 0 && (!colind || !values))) throw std::invalid_argument("null argument");
    *info = trl_solve_info{};
    auto ctx = Context::create(device, nullptr);
    ctx->set_batching(p->batching != 0);
    const auto h = ctx->handle();
    double h2d = 0.0, d2h = 0.0;
    DeviceCSR<double> A64(ctx, n, nnz, rowptr, colind, values);
    h2d += 4.0 * (n + 1) + 12.0 * nnz;
    std::unique_ptr<DeviceCSR<float>> A32;
    if (p->mode != TRL_MODE_FP64) {
      A32 = std::make_unique<DeviceCSR<float>>(ctx, n, nnz, rowptr, colind, values);
      h2d += 4.0 * (n + 1) + 8.0 * nnz;
    }
    DeviceBuffer X0d(ctx, sizeof(double) * static_cast<std::size_t>(n) * p->bs);
    ctx->check(trl_cuda_memcpy(h, X0d.get(), X0, X0d.bytes(), TRL_H2D), "upload X0");
    h2d += static_cast<double>(X0d.bytes());
    DeviceBuffer E;
    if (evecs) E = DeviceBuffer(ctx, sizeof(double) * static_cast<std::size_t>(n) * p->nev);
    trl_solve_params q = *p;
    if (evecs || resid) q.want_vectors = 1;
    int st = dispatch(ctx, q, A64.desc(), A32 ? A32->desc() : nullptr, static_cast<const double*>(X0d.get()), evals, evecs ? static_cast<double*>(E.get()) : nullptr, resid,
                      info);
    if (st) return st;
    d2h += sizeof(double) * p->nev;
    if (evecs) {
      ctx->check(trl_cuda_memcpy(h, evecs, E.get(), E.bytes(), TRL_D2H), "download eigenvectors");
      d2h += static_cast<double>(E.bytes());
    }
    info->h2d_bytes = h2d;
    info->d2h_bytes = d2h;
    return TRL_OK;
  }
  catch (const std::invalid_argument& e) {
    return fail(e, TRL_EINVAL);
  }
  catch (const std::exception& e) {
    const std::string w = e.what();
    return fail(e, w.find("Cholesky") != std::string::npos ? TRL_ECHOLESKY : (w.find("Eigendecomposition") != std::string::npos ? TRL_EEIGEN : TRL_ECUDA));
  }
}

} // extern "C"
