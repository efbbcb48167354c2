// TEST INFRASTRUCTURE ONLY — part of the CPU oracle. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py may build, load or run anything under oracle/.
//
// CSR operator on the reference OpenMP backend. The reference applies its sparse operator
// either through Eigen (examples/openmp/csrevp.hh:36-44, lower-triangle selfadjointView) or
// through a row-per-work-item kernel on full-storage CSR (examples/sycl/csrevp.hh:159-187).
// Eigen is not installed here, so this follows the full-storage CSR semantics of the latter:
// Y[r,:] = sum_k val[k] * X[col[k],:] over the row's entries, parallelised over rows.
// The optional shift (Y = alpha*A*X + beta*X) turns "smallest eigenvalues" into "largest
// magnitude" for the reference's |theta|-descending ordering (evp_base.hh:103).
#pragma once

#include <trl/impl/openmp/evp_base.hh>

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace trl_oracle {

template <class T, unsigned int bs>
class CSREVP : public trl::openmp::EVPBase<T, bs> {
public:
  using Base = trl::openmp::EVPBase<T, bs>;
  using BlockView = typename Base::BlockView;

  CSREVP(std::size_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, double alpha = 1.0, double beta = 0.0)
      : Base(n)
      , rowptr_(rowptr)
      , colind_(colind)
      , values_(values)
      , alpha_(alpha)
      , beta_(beta)
  {
  }

  void apply(BlockView X, BlockView Y) override
  {
    const std::size_t n = this->size();
    const T* x = X.data_;
    T* y = Y.data_;
#pragma omp parallel for schedule(dynamic, 512)
    for (std::size_t r = 0; r < n; ++r) {
      T acc[bs] = {};
      for (std::int32_t k = rowptr_[r]; k < rowptr_[r + 1]; ++k) {
        const T v = static_cast<T>(values_[k]);
        const T* xr = x + static_cast<std::size_t>(colind_[k]) * bs;
#pragma omp simd
        for (unsigned j = 0; j < bs; ++j) acc[j] += v * xr[j];
      }
      for (unsigned j = 0; j < bs; ++j) y[r * bs + j] = static_cast<T>(alpha_) * acc[j] + static_cast<T>(beta_) * x[r * bs + j];
    }
  }

  /// The driver calls solve_small_dense once per restart cycle (lanczos.hh:85): the times of
  /// those calls mark the end of each cycle (for the CPU baseline's per-cycle timing).
  std::size_t solve_small_dense(const typename Base::BlockMatrix& B, typename Base::BlockMatrixBlockView beta, std::size_t nev) override
  {
    const std::size_t r = Base::solve_small_dense(B, beta, nev);
    cycle_ends.push_back(std::chrono::steady_clock::now());
    return r;
  }

  std::vector<std::chrono::steady_clock::time_point> cycle_ends;

private:
  const std::int32_t* rowptr_;
  const std::int32_t* colind_;
  const double* values_;
  double alpha_, beta_;
};

/// The generalised eigenproblem of the reference's example (examples/openmp/csrevp.hh:52-109)
/// with its operator given explicitly as a CSR matrix (there: (A - sigma B)^{-1} B through
/// Eigen's SparseLU, which is not available here) and its inner product dot = V^T (B W)
/// (:89-97), B a CSR matrix. The restated EVPBase orthonormalizes through dot(), as the
/// reference's does (evp_base.hh:43-50).
template <class T, unsigned int bs>
class CSRMInnerEVP : public CSREVP<T, bs> {
public:
  using Base = CSREVP<T, bs>;
  using BlockView = typename Base::BlockView;

  CSRMInnerEVP(std::size_t n, const std::int32_t* rowptr, const std::int32_t* colind, const double* values, const std::int32_t* mrow, const std::int32_t* mcol,
               const double* mval)
      : Base(n, rowptr, colind, values)
      , M_(n, mrow, mcol, mval)
      , tmp_(n * bs)
  {
  }

  void dot(BlockView V, BlockView W, typename Base::BlockMatrixBlockView R) override
  {
    BlockView Tview(tmp_.data(), this->size());
    M_.apply(W, Tview);
    V.dot(Tview, R);
  }

private:
  CSREVP<T, bs> M_;
  std::vector<T> tmp_;
};

} // namespace trl_oracle
