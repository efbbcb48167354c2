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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

using trl::cuda::Context;
using trl::cuda::DeviceBuffer;
using trl::cuda::DeviceCSR;
using trl::cuda::SellOp;

static_assert(trl::Eigenproblem<trl::cuda::CSREVP<double, 8>>);
static_assert(trl::Eigenproblem<trl::cuda::CSREVP<float, 8>>);
static_assert(trl::ReorthogonalizationStrategy<trl::cuda::BlockCGS2, trl::cuda::CSREVP<double, 4>, trl::cuda::BlockMultivector<double, 4>>);
static_assert(trl::ReorthogonalizationStrategy<trl::cuda::BlockCGSPartial, trl::cuda::CSREVP<double, 4>, trl::cuda::BlockMultivector<double, 4>>);

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
PhaseOut run_phase(const std::shared_ptr<Context>& ctx, const trl_csr* A, const std::shared_ptr<const SellOp>& op, const trl_solve_params& p, unsigned max_restarts, double tol,
                   const Storage* X0, unsigned kx, Storage* ritz_out)
{
  using EVP = trl::cuda::CSREVP<Storage, bs>;
  auto Adev = DeviceCSR<Storage>::wrap(A->n, A->nnz, A->rowptr, A->colind, static_cast<const Storage*>(A->values));
  auto evp = std::make_shared<EVP>(ctx, std::move(Adev), p.alpha, p.beta, op);
  evp->set_cholqr_passes(p.cholqr_passes);
  evp->set_full_eigenvectors(p.small_eigen_full != 0);
  if (p.partial_threshold > 0.0) evp->set_partial_threshold(p.partial_threshold);
  evp->set_partial_pairs(p.partial_pairs != 0);
  evp->set_min_eigenvectors(static_cast<std::size_t>(kx) * bs); // the Ritz vectors formed below
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
PhaseOut run_phase_r(const std::shared_ptr<Context>& ctx, const trl_csr* A, const std::shared_ptr<const SellOp>& op, const trl_solve_params& p, unsigned max_restarts, double tol,
                     const Storage* X0, unsigned kx, Storage* ritz_out)
{
  switch (p.reorth) {
  case TRL_REORTH_MGS: return run_phase<Storage, bs, trl::ModifiedGS>(ctx, A, op, p, max_restarts, tol, X0, kx, ritz_out);
  case TRL_REORTH_CGS2: return run_phase<Storage, bs, trl::cuda::BlockCGS2>(ctx, A, op, p, max_restarts, tol, X0, kx, ritz_out);
  case TRL_REORTH_CGS1: return run_phase<Storage, bs, trl::cuda::BlockCGS1>(ctx, A, op, p, max_restarts, tol, X0, kx, ritz_out);
  case TRL_REORTH_PARTIAL: return run_phase<Storage, bs, trl::cuda::BlockCGSPartial>(ctx, A, op, p, max_restarts, tol, X0, kx, ritz_out);
  default: return run_phase<Storage, bs, trl::cuda::BlockCGSIfNeeded>(ctx, A, op, p, max_restarts, tol, X0, kx, ritz_out);
  }
}

// ---- FP64 refinement of the mixed mode by Chebyshev-filtered subspace iteration ---------
//
// The FP32 phase hands over nev/bs + 2 blocks of Ritz vectors (one block more than the
// thick restart keeps) accurate to about fp32_tol. Their span already holds the wanted
// eigenvectors up to that accuracy; what is left is to damp the components along the rest
// of the spectrum. A Chebyshev polynomial of degree d on the interval [a, b] that holds
// every unwanted eigenvalue (a a Gershgorin bound, b the smallest kept Ritz value)
// amplifies an eigenvector with eigenvalue x > b by T_d((x - c) / e) (c, e the interval's
// centre and half-width) relative to the damped ones. The filter is applied with the
// three-term recurrence in the scaled form of Zhou & Saad (2007, "Chebyshev-filtered
// subspace iteration"), one multi-block SpMM per degree that reads the CSR stream once for
// all kept blocks. The block is re-orthonormalised whenever the spread of amplifications
// across the kept vectors reaches about 1e6 (1e3 in FP32), and a Rayleigh-Ritz step (dense
// eigenproblem of the kept vectors, FP64) follows every filter round; a round aims at two
// orders of magnitude at most. Rounds filter in FP32 (FP32 operator and vectors, half the
// bytes per degree) while the wanted residual is above what FP32 vectors resolve, then in
// FP64. The Ritz pairs are final when every wanted pair has ||op x - theta x|| / |theta| <
// tol (the driver's convergence test, evp_base.hh:128-147). No Krylov basis is built, so
// there is no reorthogonalisation against a growing basis: each degree costs one CSR pass
// plus the kept blocks' gathers and stores.

struct RefineOut {
  bool applicable = false; // false: the Lanczos refinement takes over (the filter does not apply, or is predicted slower)
  bool converged = false;
  unsigned rounds = 0;
  unsigned degree = 0;   // total filter degree (FP32 and FP64 rounds)
  unsigned degree32 = 0; // of which FP32
  double predicted_s = 0.0; // TRL_REFINE_AUTO: the filter's predicted time
  std::vector<double> evals; // Ritz values of the last Rayleigh-Ritz step, |theta| descending
};

template <unsigned bs>
class ChebyshevRefinement {
public:
  /// A: the FP64 operator (CSR, for its Gershgorin bounds) and op64 its prepared copy;
  /// op32 (may be null): the prepared FP32 copy, for the FP32 filter rounds.
  ChebyshevRefinement(std::shared_ptr<Context> ctx, const trl_csr* A, std::shared_ptr<const SellOp> op64, std::shared_ptr<const SellOp> op32, const trl_solve_params& p,
                      unsigned kr)
      : ctx_(std::move(ctx))
      , h_(ctx_->handle())
      , A_(A)
      , op64_(std::move(op64))
      , op32_(std::move(op32))
      , p_(p)
      , kr_(kr)
      , n_(A->n)
      , blk_(static_cast<std::size_t>(A->n) * bs)
      , Y_(ctx_, sizeof(double) * blk_ * kr)
      , AX_(ctx_, sizeof(double) * blk_ * kr)
      , AXr_(ctx_, sizeof(double) * blk_ * kr)
      , R_(ctx_, sizeof(double) * blk_)
      , T_(ctx_, sizeof(double) * kr * kr * bs * bs)
      , C_(ctx_, sizeof(double) * kr * bs * bs)
      , Z_(ctx_, sizeof(double) * kr * kr * bs * bs)
      , ev_(ctx_, sizeof(double) * kr * bs)
      , small_(ctx_, sizeof(double) * 4 * bs * bs)
      , X32_(ctx_, op32_ ? sizeof(float) * blk_ * kr : 0)
      , Y32_(ctx_, op32_ ? sizeof(float) * blk_ * kr : 0)
  {
  }

  /// X: kr blocks (device, FP64) of approximate Ritz vectors; on exit the Ritz vectors of
  /// the last Rayleigh-Ritz step, |theta| descending. lanczos_estimate_s > 0: before the
  /// first filter round the refinement compares its own predicted time with this estimate of
  /// the Lanczos refinement's and gives up (applicable = false, X the Rayleigh-Ritz vectors)
  /// when the filter would take longer. The decision is made once: neither estimate is
  /// reliable enough to stop a running filter (on the 512^2 generalised problem the Lanczos
  /// estimate was 0.037 s against 8 s measured, while the filter finished in 0.55 s).
  RefineOut run(double* X, double lanczos_estimate_s = 0.0)
  {
    RefineOut out;
    double lo = 0.0, hi = 0.0;
    ctx_->check(trl_cuda_csr_gershgorin(h_, A_, p_.alpha, p_.beta, &lo, &hi), "refine bounds");
    double* cur = X;
    double* spare = static_cast<double*>(Y_.get());
    {
      EventTimer t(static_cast<cudaStream_t>(trl_cuda_stream(h_)));
      t.start();
      orthonormalize(cur);
      t_orth_ = t.stop(); // the cost of one re-orthonormalisation inside the filter
    }
    const unsigned N = kr_ * bs;
    bool use32 = op32_ != nullptr;
    double prev_res = 0.0; // residual at the start of the last FP32 round
    for (unsigned round = 0; round < kMaxRounds; ++round) {
      std::vector<double> theta = rayleigh_ritz(cur, spare); // cur <- Ritz vectors (in spare, swapped)
      std::swap(cur, spare);
      out.rounds = round + 1;
      out.evals = theta;
      const double res = wanted_residual(cur, theta);
      if (res < p_.tol) {
        out.applicable = out.converged = true;
        return finish(out, cur, X);
      }
      if (round + 1 == kMaxRounds) break; // leave the last Rayleigh-Ritz vectors in place
      // orientation. Kept Ritz values on one side of zero: filter s * op (s the sign of the
      // kept values) on the damped interval [a, b], a the far Gershgorin bound, b the kept
      // value nearest the rest of the spectrum. Kept values on both sides of zero (the
      // largest-magnitude eigenvalues of an indefinite operator): the interval [-b, b], b the
      // smallest kept |theta|, centred at zero, so that T_d(op / b) amplifies both ends alike
      // (|T_d(x / b)| grows with |x| outside it).
      double tmin = theta[0], tmax = theta[0];
      for (double t : theta) {
        tmin = std::min(tmin, t);
        tmax = std::max(tmax, t);
      }
      const bool one_sided = tmin > 0.0 || tmax < 0.0;
      const double s = one_sided && tmax < 0.0 ? -1.0 : 1.0;
      const double b = one_sided ? (s > 0 ? tmin : -tmax) : std::abs(theta[N - 1]);
      const double a = one_sided ? (s > 0 ? lo : -hi) : -b;
      const double top = std::abs(theta[0]);                                          // largest |theta|
      const double worst = std::abs(theta[std::min<std::size_t>(p_.nev, N) - 1]);     // smallest wanted
      const double c = 0.5 * (a + b), e = 0.5 * (b - a);
      if (!(e > 0.0) || !(worst > b)) return finish(out, cur, X); // not applicable
      const double xw = (worst - c) / e, xt = (top - c) / e;
      const double rw = std::acosh(xw), rt = std::acosh(std::max(xt, xw));
      if (round == 0 && lanczos_estimate_s > 0.0) {
        // predicted filter time: the degrees to reach the tolerance at the predicted rate
        // (optimistic early on, so this errs towards the filter) times one degree, measured
        // as the Rayleigh-Ritz step's multi-block SpMM (each degree is one such SpMM plus a
        // share of re-orthonormalisation and Rayleigh-Ritz steps, counted as 25% more).
        // The two-sided filter is held to a 4x margin: on an indefinite spectrum the
        // interval [-b, b] leaves unwanted eigenvalues close to both of its ends, and its
        // early rate estimate was up to 25x too high (Zipf pattern, 4.2M rows, block size 4:
        // predicted 6.3 s, took 160 s), against about 5x for a one-sided filter.
        // A degree also carries its share of the re-orthonormalisations, one per chunk of
        // degrees (the FP64 chunk length below).
        const double degrees = std::log(std::max(res / p_.tol, 1.0)) / rw;
        const double chunk64 = rt - rw > 0.0 ? std::clamp(std::log(1e6) / (rt - rw), 4.0, static_cast<double>(kMaxDegree)) : static_cast<double>(kMaxDegree);
        out.predicted_s = (one_sided ? 1.25 : 5.0) * degrees * (t_spmm_ + t_orth_ / chunk64);
        if (out.predicted_s > lanczos_estimate_s) return finish(out, cur, X); // not applicable: the Lanczos refinement is cheaper
      }
      // FP32 rounds while the residual is above what FP32 vectors resolve and FP32 rounds
      // still make progress (a round that gains less than 1.05x has met the FP32 floor)
      if (use32 && prev_res > 0.0 && !(res < prev_res / 1.05)) use32 = false;
      if (use32 && !(res > kFp32Floor)) use32 = false;
      prev_res = use32 ? res : 0.0;
      // degree: reduce the worst wanted residual to a tenth of the tolerance (FP32 rounds:
      // to the FP32 target), at most two orders of magnitude per round. The predicted rate
      // acosh((worst - c) / e) assumes accurate Ritz values; early on the smallest kept one
      // (b) is too low and the rate several times too high, so a round undershoots and the
      // next Rayleigh-Ritz step (a few ms) re-estimates, instead of one long round
      // overshooting. A round runs kMinDegree degrees at least unless fewer finish the job,
      // so that early rounds are not dominated by their Rayleigh-Ritz step.
      const double target = use32 ? std::max(0.1 * p_.tol, kFp32Target) : 0.1 * p_.tol;
      const double need_all = std::log(2.0 * std::max(res / target, 2.0));
      const double need = std::min(need_all, std::log(100.0));
      // (degrees are clamped in double: rw -> 0 as the smallest wanted value nears b)
      const double dmax = static_cast<double>(kMaxDegree);
      const double d_all = std::min(std::ceil(need_all / rw), dmax);
      const double d_need = std::min(std::ceil(need / rw), dmax);
      const unsigned d = static_cast<unsigned>(std::clamp(std::max(d_need, std::min(static_cast<double>(kMinDegree), d_all)), 8.0, dmax));
      // chunk length: re-orthonormalise before the spread of amplifications exceeds ~1e6
      // (~1e3 in FP32, whose rounding would otherwise swamp the least amplified vectors)
      const double spread = rt - rw;
      const double chunk_d = spread > 0.0 ? std::log(use32 ? 1e3 : 1e6) / spread : static_cast<double>(d);
      const unsigned chunk = static_cast<unsigned>(std::clamp(chunk_d, 4.0, static_cast<double>(d)));
      unsigned done = 0;
      if (trace_)
        std::fprintf(stderr, "refine round %u fp32 %d res %.3e degree %u rate %.4f chunk %u b %.6f worst %.6f host %.1f ms\n", round, static_cast<int>(use32), res, d, rw, chunk, b,
                     worst, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count());
      if (use32) {
        float* c32 = static_cast<float*>(X32_.get());
        float* s32 = static_cast<float*>(Y32_.get());
        ctx_->check(trl_cuda_convert(h_, TRL_F32, c32, TRL_F64, cur, static_cast<std::int64_t>(blk_) * kr_), "refine narrow");
        while (done < d) {
          const unsigned L = std::min(chunk, d - done);
          if (filter(*op32_, c32, s32, L, s, c, e, top) == s32) std::swap(c32, s32);
          orthonormalize(c32);
          done += L;
        }
        ctx_->check(trl_cuda_convert(h_, TRL_F64, cur, TRL_F32, c32, static_cast<std::int64_t>(blk_) * kr_), "refine widen");
        orthonormalize(cur);
        out.degree32 += d;
      }
      else {
        while (done < d) {
          const unsigned L = std::min(chunk, d - done);
          if (filter(*op64_, cur, spare, L, s, c, e, top) == spare) std::swap(cur, spare); // the filtered block is in cur
          orthonormalize(cur);
          done += L;
        }
      }
      out.degree += d;
    }
    out.applicable = true;
    return finish(out, cur, X);
  }

private:
  static constexpr unsigned kMaxRounds = 40;
  static constexpr unsigned kMaxDegree = 4000;
  static constexpr unsigned kMinDegree = 64;
  // FP32 filter rounds run while the wanted residual is above kFp32Floor and aim at
  // kFp32Target: FP32 vectors resolve ||op x - theta x|| / |theta| to about 4e-6 on the
  // 96^3 workload
  static constexpr double kFp32Floor = 2e-5;
  static constexpr double kFp32Target = 3e-6;

  std::shared_ptr<Context> ctx_;
  trl_cuda_handle h_;
  const trl_csr* A_;
  std::shared_ptr<const SellOp> op64_, op32_;
  double t_spmm_ = 0.0; // seconds of one multi-block SpMM over the kept blocks
  double t_orth_ = 0.0; // seconds of one orthonormalisation of the kept blocks
  trl_solve_params p_;
  unsigned kr_;
  std::int64_t n_;
  std::size_t blk_;
  DeviceBuffer Y_, AX_, AXr_, R_, T_, C_, Z_, ev_, small_, X32_, Y32_;
#ifdef TRL_DEBUG_TRACE
  const bool trace_ = std::getenv("TRL_REFINE_TRACE") != nullptr; // debug builds: per-round log on stderr
#else
  static constexpr bool trace_ = false;
#endif
  const std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();

  template <class T>
  T* blockp(T* base, unsigned j) const
  {
    return base + static_cast<std::size_t>(j) * blk_;
  }

  /// Leaves the current block in the caller's buffer.
  RefineOut& finish(RefineOut& out, double* cur, double* X)
  {
    if (cur != X) ctx_->check(trl_cuda_memcpy(h_, X, cur, sizeof(double) * blk_ * kr_, TRL_D2D), "refine result");
    return out;
  }

  /// Block classical Gram-Schmidt (two passes) across the kr blocks, then CholQR2 per block.
  template <class T>
  void orthonormalize(T* X)
  {
    constexpr int dt = trl::cuda::dtype_of<T>::value;
    double* G = static_cast<double*>(small_.get());
    double* R = G + bs * bs;
    for (unsigned j = 0; j < kr_; ++j) {
      if (j > 0) ctx_->check(trl_cuda_project_out(h_, dt, X, static_cast<int>(j), blockp(X, j), n_, bs, TRL_CGS_TWO, 0.0, G), "refine orthonormalize");
      ctx_->check(trl_cuda_cholqr_gram(h_, dt, blockp(X, j), n_, bs, 2, R, j > 0 ? G : nullptr), "refine orthonormalize");
    }
  }

  /// H = X^T op X (kr x kr blocks), its eigenpairs (|theta| descending), out = X Z and
  /// AXr = (op X) Z. Returns all kr*bs Ritz values.
  std::vector<double> rayleigh_ritz(double* X, double* out)
  {
    double* AX = static_cast<double*>(AX_.get());
    double* T = static_cast<double*>(T_.get());
    double* C = static_cast<double*>(C_.get());
    if (t_spmm_ == 0.0) { // the first call times one multi-block SpMM (the cost of a filter degree)
      EventTimer t(static_cast<cudaStream_t>(trl_cuda_stream(h_)));
      t.start();
      op64_->spmm(X, AX, static_cast<int>(kr_), p_.alpha, p_.beta);
      t_spmm_ = t.stop();
    }
    else
      op64_->spmm(X, AX, static_cast<int>(kr_), p_.alpha, p_.beta);
    // lower block triangle of H: column j = X^T (op X_j), blocks k >= j
    for (unsigned j = 0; j < kr_; ++j) {
      ctx_->check(trl_cuda_block_dot(h_, TRL_F64, X, static_cast<int>(kr_), blockp(AX, j), n_, bs, C), "refine Rayleigh-Ritz");
      for (unsigned k = j; k < kr_; ++k)
        ctx_->check(trl_cuda_mb_copy(h_, T + (static_cast<std::size_t>(k) * kr_ + j) * bs * bs, C + static_cast<std::size_t>(k) * bs * bs, bs, 0), "refine Rayleigh-Ritz");
    }
    const unsigned N = kr_ * bs;
    std::vector<double> theta(N);
    int nconv = 0;
    double* zero = static_cast<double*>(small_.get()) + 2 * bs * bs;
    ctx_->check(trl_cuda_mb_zero(h_, zero, bs), "refine Rayleigh-Ritz");
    ctx_->check(trl_cuda_small_eigen_partial(h_, T, static_cast<int>(kr_), bs, zero, 0, 1.0, static_cast<int>(N), static_cast<double*>(ev_.get()), static_cast<double*>(Z_.get()),
                                             theta.data(), &nconv),
                "refine Rayleigh-Ritz");
    const double* Z = static_cast<const double*>(Z_.get());
    ctx_->check(trl_cuda_block_rotate(h_, TRL_F64, X, static_cast<int>(kr_), Z, static_cast<int>(kr_), static_cast<int>(kr_), out, n_, bs), "refine Rayleigh-Ritz");
    ctx_->check(trl_cuda_block_rotate(h_, TRL_F64, AX, static_cast<int>(kr_), Z, static_cast<int>(kr_), static_cast<int>(kr_), static_cast<double*>(AXr_.get()), n_, bs),
                "refine Rayleigh-Ritz");
    return theta;
  }

  /// max over the wanted pairs of ||op x - theta x|| / |theta| (x orthonormal).
  double wanted_residual(double* X, const std::vector<double>& theta)
  {
    double* AXr = static_cast<double*>(AXr_.get());
    double* R = static_cast<double*>(R_.get());
    double* D = static_cast<double*>(small_.get()) + 3 * bs * bs;
    double* G = static_cast<double*>(small_.get());
    std::vector<double> gh(bs * bs);
    double worst = 0.0;
    const unsigned nb = (p_.nev + bs - 1) / bs;
    for (unsigned j = 0; j < nb; ++j) {
      double diag[16] = {0};
      for (unsigned c = 0; c < bs; ++c) diag[c] = theta[j * bs + c];
      ctx_->check(trl_cuda_bv_copy(h_, TRL_F64, R, blockp(AXr, j), n_, bs), "refine residual");
      ctx_->check(trl_cuda_mb_zero(h_, D, bs), "refine residual");
      ctx_->check(trl_cuda_mb_set_diagonal(h_, D, diag, bs), "refine residual");
      ctx_->check(trl_cuda_bv_mult(h_, TRL_F64, TRL_SUBTRACT, blockp(X, j), D, R, n_, bs), "refine residual");
      ctx_->check(trl_cuda_block_dot(h_, TRL_F64, R, 1, R, n_, bs, G), "refine residual");
      ctx_->check(trl_cuda_memcpy(h_, gh.data(), G, sizeof(double) * bs * bs, TRL_D2H), "refine residual");
      for (unsigned c = 0; c < bs && j * bs + c < p_.nev; ++c)
        worst = std::max(worst, std::sqrt(std::max(0.0, gh[c * bs + c])) / std::max(std::abs(theta[j * bs + c]), 1e-300));
    }
    return worst;
  }

  /// p_L(s op) X with the scaled Chebyshev recurrence on [c - e, c + e], normalised at the
  /// point `top` (the largest kept value) so that the kept components stay O(1). X and Y are
  /// the two recurrence buffers (both overwritten); returns the one holding the result.
  template <class T>
  T* filter(const SellOp& A, T* X, T* Y, unsigned L, double s, double c, double e, double top)
  {
    // s * op = s*alpha*A + s*beta*I; the recurrence needs (s*op - c) / e
    const double al = s * p_.alpha, be = s * p_.beta - c;
    double sigma = e / (top - c);
    const double tau = 2.0 / sigma;
    // Y1 = (s op - c) X * sigma / e
    A.spmm(X, Y, static_cast<int>(kr_), al * sigma / e, be * sigma / e);
    T* prev = X;
    T* curv = Y;
    for (unsigned i = 2; i <= L; ++i) {
      const double sigma2 = 1.0 / (tau - sigma);
      // Y_{i} = 2 sigma2 / e (s op - c) Y_{i-1} - sigma sigma2 Y_{i-2}, written over Y_{i-2}
      A.spmm(curv, prev, static_cast<int>(kr_), 2.0 * sigma2 / e * al, 2.0 * sigma2 / e * be, -sigma * sigma2, prev);
      std::swap(prev, curv);
      sigma = sigma2;
    }
    return curv;
  }
};

template <unsigned bs>
int solve_device(const std::shared_ptr<Context>& ctx, const trl_solve_params& p, const trl_csr* A64, const trl_csr* A32, const double* X0, double* evals_host,
                 double* evecs_dev, double* resid_host, trl_solve_info* info)
{
  const auto h = ctx->handle();
  const std::int64_t n = A64->n;
  const unsigned kx = (p.nev + bs - 1) / bs; // blocks of Ritz vectors to form
  const unsigned kr = p.nev / bs + 1;        // blocks the thick restart keeps (lanczos.hh:97)
  // blocks the Chebyshev refinement iterates on: one more than the restart keeps. Its cost
  // per order of magnitude is ~ blocks / acosh(1 + 2 (theta_nev - theta_last) / (theta_last -
  // a)); on the 96^3 workload (nev 32, bs 8) that is 306 for 5 blocks, 231 for 6, ~228 for 7-8.
  const unsigned kref = kr + 1;
  cudaStream_t stream = static_cast<cudaStream_t>(trl_cuda_stream(h));
  const auto launches0 = trl_cuda_launch_count(h);

  EventTimer total(stream), phase(stream);
  total.start();
#ifdef TRL_DEBUG_TRACE
  // debug builds with TRL_REFINE_TRACE set: host timestamps of the solve's stages on stderr
  const bool trace = std::getenv("TRL_REFINE_TRACE") != nullptr;
#else
  constexpr bool trace = false;
#endif
  const auto host0 = std::chrono::steady_clock::now();
  const auto stage = [&](const char* what) {
    if (trace) std::fprintf(stderr, "solve %s host %.1f ms\n", what, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host0).count());
  };
  DeviceBuffer X64(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs * std::max(kx, kref));
  PhaseOut out;
  double t32 = 0.0;
  // the operator prepared for this block size (sliced-ELL copies, built on the device inside
  // the timed solve): FP64 for the FP64 solve, the refinement and the residuals, FP32 for the
  // FP32 phases
  if (p.mode != TRL_MODE_FP64 && !A32) throw std::invalid_argument("FP32 and mixed modes need the FP32 copy of the operator");
  const bool need64 = p.mode != TRL_MODE_FP32 || p.want_vectors;
  const std::shared_ptr<const SellOp> op64 = need64 ? std::make_shared<const SellOp>(ctx, A64, static_cast<int>(bs)) : nullptr;
  const std::shared_ptr<const SellOp> op32 = p.mode != TRL_MODE_FP64 ? std::make_shared<const SellOp>(ctx, A32, static_cast<int>(bs)) : nullptr;
  stage("operators prepared");

  if (p.mode == TRL_MODE_FP64) {
    out = run_phase_r<double, bs>(ctx, A64, op64, p, p.max_restarts, p.tol, X0, p.want_vectors ? kx : 0, static_cast<double*>(X64.get()));
  }
  else {
    DeviceBuffer X32(ctx, sizeof(float) * static_cast<std::size_t>(n) * bs * std::max(kx, kref));
    DeviceBuffer X0f(ctx, sizeof(float) * static_cast<std::size_t>(n) * bs);
    ctx->check(trl_cuda_convert(h, TRL_F32, X0f.get(), TRL_F64, X0, n * bs), "initial block");
    if (p.mode == TRL_MODE_FP32) {
      out = run_phase_r<float, bs>(ctx, A32, op32, p, p.max_restarts, p.tol, static_cast<const float*>(X0f.get()), kx, static_cast<float*>(X32.get()));
      ctx->check(trl_cuda_convert(h, TRL_F64, X64.get(), TRL_F32, X32.get(), n * bs * kx), "widen");
    }
    else {
      phase.start();
      trl_solve_params p32 = p;
      if (p.fp32_ncv) p32.ncv = p.fp32_ncv;
      const unsigned k32 = std::min(kref, p32.ncv / bs); // Ritz blocks the FP32 phase hands over
      PhaseOut o32 = run_phase_r<float, bs>(ctx, A32, op32, p32, p.max_restarts, p.fp32_tol, static_cast<const float*>(X0f.get()), k32, static_cast<float*>(X32.get()));
      t32 = phase.stop();
      stage("fp32 phase done");
      info->restarts_fp32 = o32.restarts;
      info->n_op_apply_fp32 = o32.applies;
      // FP64 refinement: widen the kept FP32 Ritz vectors and start the FP64 solve from a
      // seeded random combination of them (the start block then carries every wanted
      // direction to FP32 accuracy).
      ctx->check(trl_cuda_convert(h, TRL_F64, X64.get(), TRL_F32, X32.get(), n * bs * k32), "widen");
      bool refined = false;
      if (p.refine == TRL_REFINE_CHEBYSHEV || p.refine == TRL_REFINE_AUTO) {
        ChebyshevRefinement<bs> cheb(ctx, A64, op64, p.refine_fp32 ? op32 : nullptr, p, k32);
        stage("refinement buffers allocated");
        // TRL_REFINE_AUTO: the Lanczos refinement is estimated from the FP32 phase, which
        // took t32 to gain log(1/fp32_tol) orders; the FP64 phase gains log(1/tol) orders at
        // about 1.5 times the FP32 cost per step
        const double lanczos_s = p.refine == TRL_REFINE_AUTO ? 1.5 * t32 * std::log(1.0 / p.tol) / std::log(1.0 / std::max(p.fp32_tol, 1e-7)) : 0.0;
        const RefineOut r = cheb.run(static_cast<double*>(X64.get()), lanczos_s);
        stage("refinement done");
        info->refine_predicted_s = r.predicted_s;
        info->refine_lanczos_estimate_s = lanczos_s;
        // the filter's work, also when it handed over to the Lanczos refinement
        info->refine_rounds = r.rounds;
        info->refine_degree = r.degree;
        info->refine_degree_fp32 = r.degree32;
        if (r.applicable) {
          info->refine_used = TRL_REFINE_CHEBYSHEV;
          refined = true;
          out.converged = r.converged;
          out.restarts = 0;
          out.applies = 0;
          out.evals = r.evals;
        }
      }
      if (!refined) {
      info->refine_used = TRL_REFINE_LANCZOS;
      std::vector<double> G(static_cast<std::size_t>(kr) * bs * bs);
      std::mt19937 rng(p.seed);
      std::normal_distribution<double> dist;
      for (auto& g : G) g = dist(rng);
      DeviceBuffer Gd(ctx, sizeof(double) * G.size());
      ctx->check(trl_cuda_memcpy(h, Gd.get(), G.data(), sizeof(double) * G.size(), TRL_H2D), "refine coefficients");
      DeviceBuffer V0(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs);
      ctx->check(trl_cuda_block_rotate(h, TRL_F64, X64.get(), static_cast<int>(kr), static_cast<const double*>(Gd.get()), 1, 1, V0.get(), n, bs), "refine start");
      ctx->check(trl_cuda_synchronize(h), "refine start");
      out = run_phase_r<double, bs>(ctx, A64, op64, p, p.refine_max_restarts, p.tol, static_cast<const double*>(V0.get()), p.want_vectors ? kx : 0,
                                    static_cast<double*>(X64.get()));
      }
    }
  }
  info->converged = out.converged ? 1 : 0;
  info->restarts = out.restarts;
  info->n_op_apply = out.applies;
  info->seconds_fp32 = t32;
  for (unsigned c = 0; c < p.nev; ++c) evals_host[c] = c < out.evals.size() ? out.evals[c] : 0.0;

  stage("eigenpairs found");
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
      op64->spmm(Xj, R.get(), 1, p.alpha, p.beta);
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
  stage("residuals done");
  info->kernel_launches = trl_cuda_launch_count(h) - launches0;
  return TRL_OK;
}

// ---- matrix-weighted inner product (K x = lambda M x through an M-self-adjoint operator) --

template <unsigned bs, class Reorth>
int solve_minner_phase(const std::shared_ptr<Context>& ctx, const trl_solve_params& p, const trl_csr* op, const trl_csr* M, const double* X0, double* evals_host,
                       double* evecs_dev, double* resid_host, trl_solve_info* info)
{
  using EVP = trl::cuda::MInnerCSREVP<double, bs>;
  const auto h = ctx->handle();
  const std::int64_t n = op->n;
  const unsigned kx = (p.nev + bs - 1) / bs;
  cudaStream_t stream = static_cast<cudaStream_t>(trl_cuda_stream(h));
  EventTimer total(stream);
  total.start();
  const auto launches0 = trl_cuda_launch_count(h);
  auto opd = DeviceCSR<double>::wrap(op->n, op->nnz, op->rowptr, op->colind, static_cast<const double*>(op->values));
  auto Md = DeviceCSR<double>::wrap(M->n, M->nnz, M->rowptr, M->colind, static_cast<const double*>(M->values));
  auto evp = std::make_shared<EVP>(ctx, std::move(opd), std::move(Md), p.alpha, p.beta);
  evp->set_cholqr_passes(p.cholqr_passes);
  evp->set_full_eigenvectors(p.small_eigen_full != 0);
  evp->set_min_eigenvectors(static_cast<std::size_t>(kx) * bs);
  trl::EigensolverParams ep{.nev = p.nev, .ncv = p.ncv, .max_restarts = p.max_restarts, .tolerance = p.tol};
  trl::BlockLanczos<EVP, Reorth> lanczos(evp, ep);
  auto V0 = lanczos.initial_block();
  ctx->flush();
  ctx->check(trl_cuda_memcpy(h, V0.data_, X0, sizeof(double) * static_cast<std::size_t>(n) * bs, TRL_D2D), "initial block");
  const auto res = lanczos.solve();
  ctx->flush();
  info->converged = res.converged ? 1 : 0;
  info->restarts = res.iterations;
  info->n_op_apply = res.n_op_apply;
  const auto ev = evp->get_current_eigenvalues();
  for (unsigned c = 0; c < p.nev; ++c) evals_host[c] = c < ev.size() ? ev[c] : 0.0;
  if (p.want_vectors) {
    DeviceBuffer X(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs * kx);
    auto& V = lanczos.get_basis();
    const auto& Y = evp->get_current_eigenvectors();
    ctx->check(trl_cuda_block_rotate(h, TRL_F64, V.data(), static_cast<int>(p.ncv / bs), Y.data(), static_cast<int>(Y.block_cols()), static_cast<int>(kx), X.get(), n, bs),
               "ritz vectors");
    // residuals ||op x - theta x|| / ||op||_1 (Euclidean norms; x is M-normalised)
    SellOp opsell(ctx, op, static_cast<int>(bs));
    double norm1 = 0.0;
    ctx->check(trl_cuda_csr_norm1(h, op, p.alpha, p.beta, &norm1), "norm");
    info->op_norm1 = norm1;
    DeviceBuffer R(ctx, sizeof(double) * static_cast<std::size_t>(n) * bs), D(ctx, sizeof(double) * bs * bs), G(ctx, sizeof(double) * bs * bs * 2);
    std::vector<double> gh(2 * bs * bs);
    for (unsigned j = 0; j < kx; ++j) {
      const double* Xj = static_cast<const double*>(X.get()) + static_cast<std::size_t>(j) * n * bs;
      opsell.spmm(Xj, R.get(), 1, p.alpha, p.beta);
      double diag[16] = {0};
      for (unsigned c = 0; c < bs; ++c) diag[c] = (j * bs + c < p.nev) ? evals_host[j * bs + c] : 0.0;
      ctx->check(trl_cuda_mb_zero(h, static_cast<double*>(D.get()), bs), "residual");
      ctx->check(trl_cuda_mb_set_diagonal(h, static_cast<double*>(D.get()), diag, bs), "residual");
      ctx->check(trl_cuda_bv_mult(h, TRL_F64, TRL_SUBTRACT, Xj, static_cast<const double*>(D.get()), R.get(), n, bs), "residual");
      ctx->check(trl_cuda_block_dot(h, TRL_F64, R.get(), 1, R.get(), n, bs, static_cast<double*>(G.get())), "residual");
      ctx->check(trl_cuda_block_dot(h, TRL_F64, Xj, 1, Xj, n, bs, static_cast<double*>(G.get()) + bs * bs), "residual");
      ctx->check(trl_cuda_memcpy(h, gh.data(), G.get(), sizeof(double) * 2 * bs * bs, TRL_D2H), "residual");
      for (unsigned c = 0; c < bs && j * bs + c < p.nev; ++c) {
        const double r_rel = std::sqrt(std::max(0.0, gh[c * bs + c])) / std::max(std::sqrt(std::max(0.0, gh[bs * bs + c * bs + c])), 1e-300);
        if (resid_host) resid_host[j * bs + c] = r_rel / std::max(norm1, 1e-300);
        info->max_rel_residual = std::max(info->max_rel_residual, r_rel / std::max(norm1, 1e-300));
        info->max_theta_residual = std::max(info->max_theta_residual, r_rel / std::max(std::abs(evals_host[j * bs + c]), 1e-300));
      }
    }
    if (evecs_dev) ctx->check(trl_cuda_unblock(h, static_cast<const double*>(X.get()), n, bs, static_cast<int>(p.nev), evecs_dev), "ritz vectors");
  }
  ctx->sync();
  info->seconds = total.stop();
  info->kernel_launches = trl_cuda_launch_count(h) - launches0;
  return TRL_OK;
}

template <unsigned bs>
int solve_minner_r(const std::shared_ptr<Context>& ctx, const trl_solve_params& p, const trl_csr* op, const trl_csr* M, const double* X0, double* ev, double* evecs, double* resid,
                   trl_solve_info* info)
{
  switch (p.reorth) {
  case TRL_REORTH_MGS: return solve_minner_phase<bs, trl::ModifiedGS>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case TRL_REORTH_CGS1: return solve_minner_phase<bs, trl::cuda::BlockCGS1>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case TRL_REORTH_CGS2: return solve_minner_phase<bs, trl::cuda::BlockCGS2>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case TRL_REORTH_PARTIAL: return solve_minner_phase<bs, trl::cuda::BlockCGSPartial>(ctx, p, op, M, X0, ev, evecs, resid, info);
  default: return solve_minner_phase<bs, trl::cuda::BlockCGSIfNeeded>(ctx, p, op, M, X0, ev, evecs, resid, info);
  }
}

int dispatch_minner(const std::shared_ptr<Context>& ctx, const trl_solve_params& p, const trl_csr* op, const trl_csr* M, const double* X0, double* ev, double* evecs,
                    double* resid, trl_solve_info* info)
{
  switch (p.bs) {
  case 1: return solve_minner_r<1>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case 2: return solve_minner_r<2>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case 4: return solve_minner_r<4>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case 8: return solve_minner_r<8>(ctx, p, op, M, X0, ev, evecs, resid, info);
  case 16: return solve_minner_r<16>(ctx, p, op, M, X0, ev, evecs, resid, info);
  default: throw std::invalid_argument("unsupported block size " + std::to_string(p.bs));
  }
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

} // namespace

namespace trl_solver_detail {
int set_error(int status, const char* msg)
{
  g_err = msg;
  return status;
}
} // namespace trl_solver_detail

namespace {

// trl_solve_csr_host's context on each device: created by the first call and kept until
// the process exits, so that its memory pool keeps the solve's buffers reserved between
// calls (allocating and freeing a solve's 4-6 GB each call cost up to a second of host time
// on B200). Calls on one device are serialised.
struct HostContext {
  std::mutex m;
  std::shared_ptr<Context> ctx;
};

HostContext& host_context(int device)
{
  static std::mutex registry_lock;
  static auto* registry = new std::map<int, std::unique_ptr<HostContext>>(); // never destroyed: outlives static teardown
  std::lock_guard<std::mutex> g(registry_lock);
  auto& slot = (*registry)[device];
  if (!slot) slot = std::make_unique<HostContext>();
  return *slot;
}

void validate(const trl_solve_params* p)
{
  if (!p) throw std::invalid_argument("null params");
  if (p->mode < TRL_MODE_FP64 || p->mode > TRL_MODE_MIXED) throw std::invalid_argument("bad mode");
  if (p->ncv % p->bs != 0) throw std::invalid_argument("ncv must be a multiple of the block size");
  if (p->fp32_ncv % p->bs != 0) throw std::invalid_argument("fp32_ncv must be a multiple of the block size");
  if (p->cholqr_passes < 1 || p->cholqr_passes > 4) throw std::invalid_argument("cholqr_passes must be in [1, 4]");
  if (p->reorth < TRL_REORTH_MGS || p->reorth > TRL_REORTH_PARTIAL) throw std::invalid_argument("bad reorth strategy");
  if (!(p->partial_threshold >= 0.0)) throw std::invalid_argument("partial_threshold must be >= 0");
  if (p->refine != TRL_REFINE_LANCZOS && p->refine != TRL_REFINE_CHEBYSHEV && p->refine != TRL_REFINE_AUTO) throw std::invalid_argument("bad refinement");
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
  p->reorth = TRL_REORTH_PARTIAL; // 96^3 workload: 1.25 s against 2.53 s for TRL_REORTH_CGS_IFNEEDED, same restarts and residuals
  p->cholqr_passes = 2;
  p->fp32_tol = 3e-3; // 96^3 workload: 4 FP32 restarts, then filter degree ~1170 of which ~640 in FP32 (0.42 s; 1e-2 and 3e-2 within noise, 1e-3: 0.53 s)
  p->refine_max_restarts = 1000;
  p->want_vectors = 1;
  p->batching = 1;
  p->seed = 42;
  p->refine = TRL_REFINE_AUTO;
  p->refine_fp32 = 1;
  p->partial_pairs = 1; // 96^3 workload: 242 of 3058 steps projected, 1.25 s; 822 steps and 1.56 s without
}

const char* trl_solver_last_error(void) { return g_err.c_str(); }

int trl_solve_csr_minner_device(trl_cuda_handle h, const trl_solve_params* p, const trl_csr* op, const trl_csr* M, const double* X0, double* evals_host, double* evecs_dev,
                                double* resid_host, trl_solve_info* info)
{
  try {
    validate(p);
    if (!h || !op || !M || !X0 || !evals_host || !info) throw std::invalid_argument("null argument");
    if (p->mode != TRL_MODE_FP64) throw std::invalid_argument("the M inner product runs in FP64 only");
    if (op->value_dtype != TRL_F64 || M->value_dtype != TRL_F64) throw std::invalid_argument("operator and M must have FP64 values");
    if (M->n != op->n) throw std::invalid_argument("M must have the operator's size");
    *info = trl_solve_info{};
    auto ctx = Context::borrow(h);
    ctx->set_batching(p->batching != 0);
    return dispatch_minner(ctx, *p, op, M, X0, evals_host, evecs_dev, resid_host, info);
  }
  catch (const std::invalid_argument& e) {
    return fail(e, TRL_EINVAL);
  }
  catch (const trl::cuda::out_of_device_memory& e) {
    return fail(e, TRL_ENOMEM);
  }
  catch (const trl::cuda::device_timeout& e) {
    return fail(e, TRL_ETIMEOUT);
  }
  catch (const std::exception& e) {
    const std::string w = e.what();
    return fail(e, w.find("Cholesky") != std::string::npos ? TRL_ECHOLESKY : (w.find("Eigendecomposition") != std::string::npos ? TRL_EEIGEN : TRL_ECUDA));
  }
}

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
  catch (const trl::cuda::out_of_device_memory& e) {
    return fail(e, TRL_ENOMEM);
  }
  catch (const trl::cuda::device_timeout& e) {
    return fail(e, TRL_ETIMEOUT);
  }
  catch (const std::exception& e) {
    const std::string w = e.what();
    return fail(e, w.find("Cholesky") != std::string::npos ? TRL_ECHOLESKY : (w.find("Eigendecomposition") != std::string::npos ? TRL_EEIGEN : TRL_ECUDA));
  }
}

int trl_solve_csr_host(const trl_solve_params* p, int device, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind, const double* values, const double* X0,
                       double* evals, double* evecs, double* resid, trl_solve_info* info)
{
  HostContext* hc = nullptr;
  std::unique_lock<std::mutex> lock;
  try {
    validate(p);
    if (!rowptr || !X0 || !evals || !info || (nnz > 0 && (!colind || !values))) throw std::invalid_argument("null argument");
    *info = trl_solve_info{};
    hc = &host_context(device);
    lock = std::unique_lock<std::mutex>(hc->m);
    if (!hc->ctx) hc->ctx = Context::create(device, nullptr);
    auto ctx = hc->ctx;
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
    if (hc && lock.owns_lock()) hc->ctx.reset(); // a failed call may leave recorded work behind: start afresh
    return fail(e, TRL_EINVAL);
  }
  catch (const trl::cuda::out_of_device_memory& e) {
    if (hc && lock.owns_lock()) hc->ctx.reset();
    return fail(e, TRL_ENOMEM);
  }
  catch (const trl::cuda::device_timeout& e) {
    if (hc && lock.owns_lock()) hc->ctx.reset();
    return fail(e, TRL_ETIMEOUT);
  }
  catch (const std::exception& e) {
    if (hc && lock.owns_lock()) hc->ctx.reset();
    const std::string w = e.what();
    return fail(e, w.find("Cholesky") != std::string::npos ? TRL_ECHOLESKY : (w.find("Eigendecomposition") != std::string::npos ? TRL_EEIGEN : TRL_ECUDA));
  }
}

} // extern "C"
