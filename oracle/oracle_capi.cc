// TEST INFRASTRUCTURE ONLY — part of the CPU oracle. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py may build, load or run anything under oracle/.
//
// C entry points over the reference's own OpenMP backend, compiled in place from the
// reference headers (include/trl/eigensolvers/lanczos.hh, include/trl/impl/openmp/*.hh)
// plus the Eigen-free EVPBase restatement in oracle/shim. Every call runs the reference's
// code: BlockLanczos::solve (lanczos.hh:65-199) with its default ModifiedGS
// (reorthogonalization.hh:12-22), the BlockView kernels (impl/openmp/blockview.hh:31-201)
// and the restated orthonormalize / solve_small_dense (evp_base.hh:39-154).
#include <trl/eigensolvers/lanczos.hh>
#include <trl/eigensolvers/params.hh>
#include <trl/impl/openmp/evp_base.hh>

#include "csr_omp.hh"
#include "dense_linalg.hh"

#include <chrono>
#include <cstdio>
#include <omp.h>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>

namespace {

thread_local char g_err[512];

int fail(const char* what)
{
  std::snprintf(g_err, sizeof g_err, "%s", what);
  return 1;
}

template <unsigned bs>
class NullEVP : public trl::openmp::EVPBase<double, bs> {
public:
  using Base = trl::openmp::EVPBase<double, bs>;
  explicit NullEVP(std::size_t n)
      : Base(n)
  {
  }
  void apply(typename Base::BlockView, typename Base::BlockView) override { throw std::logic_error("NullEVP::apply"); }
};

template <unsigned bs>
int solve_csr(std::int64_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, double alpha, double beta, unsigned nev, unsigned ncv,
              unsigned max_restarts, double tol, const double* X0, double* evals_out, double* ritz_out, std::int32_t* stats, double* seconds, double* cycle_seconds)
{
  using EVP = trl_oracle::CSREVP<double, bs>;
  auto evp = std::make_shared<EVP>(static_cast<std::size_t>(n), rowptr, colind, values, alpha, beta);
  trl::EigensolverParams params{.nev = nev, .ncv = ncv, .max_restarts = max_restarts, .tolerance = tol};
  trl::BlockLanczos lanczos(evp, params);
  auto V0 = lanczos.initial_block();
  std::memcpy(V0.data_, X0, sizeof(double) * static_cast<std::size_t>(n) * bs);

  const auto t0 = std::chrono::steady_clock::now();
  const auto res = lanczos.solve();
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (cycle_seconds) { // duration of each restart cycle (cycle 1 includes the first orthonormalisation)
    auto prev = t0;
    for (std::size_t i = 0; i < evp->cycle_ends.size() && i < max_restarts; ++i) {
      cycle_seconds[i] = std::chrono::duration<double>(evp->cycle_ends[i] - prev).count();
      prev = evp->cycle_ends[i];
    }
  }
  if (stats) {
    stats[0] = res.converged ? 1 : 0;
    stats[1] = static_cast<std::int32_t>(res.iterations);
    stats[2] = static_cast<std::int32_t>(res.n_op_apply);
  }
  const auto& ev = evp->get_current_eigenvalues();
  for (std::size_t i = 0; i < ev.size() && i < ncv; ++i) evals_out[i] = ev[i];

  if (ritz_out) {
    // Ritz vectors of the basis the last projected problem was built from: x_c = sum_i V_i Y_{i, c/bs}[:, c%bs]
    const auto& Y = evp->get_current_eigenvectors();
    auto& V = lanczos.get_basis();
    const std::size_t m = ncv / bs;
    const std::size_t N = static_cast<std::size_t>(n);
#pragma omp parallel for
    for (std::size_t r = 0; r < N; ++r) {
      for (unsigned c = 0; c < nev; ++c) {
        double s = 0.0;
        for (std::size_t i = 0; i < m; ++i) {
          const double* vi = V.block_view(i).data_ + r * bs;
          const double* yb = Y.block_view(i, c / bs).data_;
          for (unsigned l = 0; l < bs; ++l) s += vi[l] * yb[l * bs + (c % bs)];
        }
        ritz_out[r * nev + c] = s;
      }
    }
  }
  return 0;
}

// The reference driver on the M-inner-product eigenproblem (trl_oracle::CSRMInnerEVP); Ritz
// vectors (M-orthonormal) into ritz_out (n x nev) when given.
template <unsigned bs>
int solve_minner(std::int64_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, const std::int32_t* mrow, const std::int32_t* mcol,
                 const double* mval, unsigned nev, unsigned ncv, unsigned max_restarts, double tol, const double* X0, double* evals_out, double* ritz_out, std::int32_t* stats)
{
  using EVP = trl_oracle::CSRMInnerEVP<double, bs>;
  auto evp = std::make_shared<EVP>(static_cast<std::size_t>(n), rowptr, colind, values, mrow, mcol, mval);
  trl::EigensolverParams params{.nev = nev, .ncv = ncv, .max_restarts = max_restarts, .tolerance = tol};
  trl::BlockLanczos lanczos(evp, params);
  std::memcpy(lanczos.initial_block().data_, X0, sizeof(double) * static_cast<std::size_t>(n) * bs);
  const auto res = lanczos.solve();
  stats[0] = res.converged ? 1 : 0;
  stats[1] = static_cast<std::int32_t>(res.iterations);
  stats[2] = static_cast<std::int32_t>(res.n_op_apply);
  const auto& ev = evp->get_current_eigenvalues();
  for (std::size_t i = 0; i < ev.size() && i < ncv; ++i) evals_out[i] = ev[i];
  if (ritz_out) {
    const auto& Y = evp->get_current_eigenvectors();
    auto& V = lanczos.get_basis();
    const std::size_t m = ncv / bs, N = static_cast<std::size_t>(n);
    for (std::size_t r = 0; r < N; ++r)
      for (unsigned c = 0; c < nev; ++c) {
        double s = 0.0;
        for (std::size_t i = 0; i < m; ++i) {
          const double* vi = V.block_view(i).data_ + r * bs;
          const double* yb = Y.block_view(i, c / bs).data_;
          for (unsigned l = 0; l < bs; ++l) s += vi[l] * yb[l * bs + (c % bs)];
        }
        ritz_out[r * nev + c] = s;
      }
  }
  return 0;
}

template <unsigned bs>
int bv_op(int op, std::int64_t n, double* X, double* Y, double* W)
{
  using BV = trl::openmp::BlockView<double, bs>;
  using MBV = trl::openmp::BlockMatrixBlockView<double, bs>;
  BV x(X, static_cast<std::size_t>(n));
  BV y(Y, static_cast<std::size_t>(n));
  MBV w(W);
  switch (op) {
  case 0: x.dot(y, w); break;              // W = X^T Y           blockview.hh:152-182
  case 1: x.mult(w, y); break;             // Y = X W             blockview.hh:104-119
  case 2: x.mult_transpose(w, y); break;   // Y = X W^T           blockview.hh:126-141
  case 3: x.mult_add(w, y); break;         // Y += X W            blockview.hh:81-97
  case 4: x.subtract_product(y, w); break; // X -= Y W            blockview.hh:189-201
  case 5: x -= y; break;                   // X -= Y              blockview.hh:69-74
  case 6: x.copy_from(y); break;           // X = Y               blockview.hh:59-63
  case 7: x.set_zero(); break;             // X = 0               blockview.hh:31-36
  default: return fail("unknown op");
  }
  return 0;
}

template <unsigned bs>
int orthonormalize(std::int64_t n, double* V, double* R)
{
  NullEVP<bs> evp(static_cast<std::size_t>(n));
  trl::openmp::BlockView<double, bs> v(V, static_cast<std::size_t>(n));
  trl::openmp::BlockMatrixBlockView<double, bs> r(R);
  evp.orthonormalize(v, r);
  return 0;
}

template <unsigned bs>
int small_dense(unsigned nblk, const double* T, const double* beta, unsigned nev, double tol, double* evals, double* evecs, std::int32_t* nconv)
{
  NullEVP<bs> evp(0);
  evp.set_tolerance(tol);
  trl::openmp::BlockMatrix<double, bs> Tm(nblk, nblk), Bm(1, 1);
  const std::size_t tsz = static_cast<std::size_t>(nblk) * nblk * bs * bs;
  // BlockMatrix storage is [br][bc][bs][bs]; block_view(0,0) points at the start.
  std::memcpy(Tm.block_view(0, 0).data_, T, tsz * sizeof(double));
  std::memcpy(Bm.block_view(0, 0).data_, beta, bs * bs * sizeof(double));
  *nconv = static_cast<std::int32_t>(evp.solve_small_dense(Tm, Bm.block_view(0, 0), nev));
  const auto& ev = evp.get_current_eigenvalues();
  std::memcpy(evals, ev.data(), ev.size() * sizeof(double));
  std::memcpy(evecs, evp.get_current_eigenvectors().block_view(0, 0).data_, tsz * sizeof(double));
  return 0;
}

template <template <unsigned> class F, class... A>
int dispatch_bs(int bs, A&&... args)
{
  switch (bs) {
  case 1: return F<1>::run(args...);
  case 2: return F<2>::run(args...);
  case 4: return F<4>::run(args...);
  case 8: return F<8>::run(args...);
  case 16: return F<16>::run(args...);
  default: return fail("unsupported block size (1, 2, 4, 8, 16)");
  }
}

template <unsigned bs>
struct SolveF {
  template <class... A>
  static int run(A... a) { return solve_csr<bs>(a...); }
};
template <unsigned bs>
struct MInnerF {
  template <class... A>
  static int run(A... a) { return solve_minner<bs>(a...); }
};
template <unsigned bs>
struct BvF {
  template <class... A>
  static int run(A... a) { return bv_op<bs>(a...); }
};
template <unsigned bs>
struct OrthF {
  template <class... A>
  static int run(A... a) { return orthonormalize<bs>(a...); }
};
template <unsigned bs>
struct SmallF {
  template <class... A>
  static int run(A... a) { return small_dense<bs>(a...); }
};

template <class Fn>
int guarded(Fn&& fn)
{
  try {
    return fn();
  }
  catch (const std::exception& e) {
    return fail(e.what());
  }
  catch (...) {
    return fail("unknown C++ exception");
  }
}

} // namespace

extern "C" {

const char* oracle_last_error() { return g_err; }

int oracle_solve_csr(int bs, std::int64_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, double alpha, double beta, unsigned nev,
                     unsigned ncv, unsigned max_restarts, double tol, const double* X0, double* evals_out, double* ritz_out, std::int32_t* stats, double* seconds,
                     double* cycle_seconds)
{
  return guarded([&] {
    return dispatch_bs<SolveF>(bs, n, rowptr, colind, values, alpha, beta, nev, ncv, max_restarts, tol, X0, evals_out, ritz_out, stats, seconds, cycle_seconds);
  });
}

int oracle_solve_csr_minner(int bs, std::int64_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, const std::int32_t* mrow,
                            const std::int32_t* mcol, const double* mval, unsigned nev, unsigned ncv, unsigned max_restarts, double tol, const double* X0,
                            double* evals_out, double* ritz_out, std::int32_t* stats)
{
  return guarded([&] { return dispatch_bs<MInnerF>(bs, n, rowptr, colind, values, mrow, mcol, mval, nev, ncv, max_restarts, tol, X0, evals_out, ritz_out, stats); });
}

int oracle_block_view_op(int bs, int op, std::int64_t n, double* X, double* Y, double* W)
{
  return guarded([&] { return dispatch_bs<BvF>(bs, op, n, X, Y, W); });
}

int oracle_orthonormalize(int bs, std::int64_t n, double* V, double* R)
{
  return guarded([&] { return dispatch_bs<OrthF>(bs, n, V, R); });
}

int oracle_solve_small_dense(int bs, unsigned nblk, const double* T, const double* beta, unsigned nev, double tol, double* evals, double* evecs, std::int32_t* nconv)
{
  return guarded([&] { return dispatch_bs<SmallF>(bs, nblk, T, beta, nev, tol, evals, evecs, nconv); });
}

int oracle_spmm(int bs, std::int64_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, double alpha, double beta, double* X, double* Y)
{
  return guarded([&]() -> int {
    switch (bs) {
#define TRL_ORACLE_SPMM(B)                                                                                                                                                                             \
  case B: {                                                                                                                                                                                            \
    trl_oracle::CSREVP<double, B> evp(static_cast<std::size_t>(n), rowptr, colind, values, alpha, beta);                                                                                              \
    evp.apply(trl::openmp::BlockView<double, B>(X, n), trl::openmp::BlockView<double, B>(Y, n));                                                                                                      \
    return 0;                                                                                                                                                                                          \
  }
      TRL_ORACLE_SPMM(1)
      TRL_ORACLE_SPMM(2)
      TRL_ORACLE_SPMM(4)
      TRL_ORACLE_SPMM(8)
      TRL_ORACLE_SPMM(16)
#undef TRL_ORACLE_SPMM
    default: return fail("unsupported block size");
    }
  });
}

int oracle_symmetric_eigen(std::int64_t n, const double* A, double* evals, double* evecs)
{
  return guarded([&] { return trl_oracle::symmetric_eigen(static_cast<std::size_t>(n), A, evals, evecs) ? 0 : fail("QR iteration did not converge"); });
}

int oracle_num_threads()
{
  int t = 1;
#pragma omp parallel
  {
#pragma omp single
    t = omp_get_num_threads();
  }
  return t;
}
}
