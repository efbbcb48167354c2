// TEST INFRASTRUCTURE ONLY — part of the CPU oracle. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py may build, load or run anything under oracle/.
//
// Eigen-free restatement of the reference's OpenMP eigenproblem base class,
// include/trl/impl/openmp/evp_base.hh:13-181 (class trl::openmp::EVPBase).
// It is found through the include path *before* the reference's own include directory,
// so the reference's headers (lanczos.hh, the OpenMP multivector/blockview/blockmatrix
// types) and its own test programs compile unchanged on top of it. Every member follows
// the reference line by line; only the three Eigen calls are replaced by the routines in
// oracle/dense_linalg.hh (Cholesky :53-55, inverse :60, SelfAdjointEigenSolver :95).
#pragma once

#include <trl/impl/openmp/multivector.hh>

#include "../../../../dense_linalg.hh"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <limits>
#include <memory>
#include <numeric>
#include <optional>
#include <span>
#include <stdexcept>
#include <vector>

namespace trl::openmp {
template <class ScalarT, unsigned int block_size>
class EVPBase {
public:
  using Scalar = ScalarT;
  constexpr static auto blocksize = block_size;

  using BlockMultivector = ::trl::openmp::BlockMultivector<Scalar, blocksize>;
  using BlockView = typename BlockMultivector::BlockView;
  using BlockMatrix = typename BlockMultivector::BlockMatrix;
  using BlockMatrixBlockView = BlockMatrix::BlockView;

  explicit EVPBase(std::size_t n)
      : N(n)
  {
    if (N > 0) Vtemp.emplace(create_multivector(N, block_size));
  }

  virtual ~EVPBase() = default;

  virtual void apply(BlockView, BlockView) = 0;

  // evp_base.hh:37
  virtual void dot(BlockView V, BlockView W, BlockMatrixBlockView R) { V.dot(W, R); }

  // evp_base.hh:39-71 — single-pass Cholesky-QR.
  virtual void orthonormalize(BlockView V, BlockMatrixBlockView R)
  {
    if constexpr (blocksize == 1) {
      this->dot(V, V, R);
      ScalarT norm = std::sqrt(R.data_[0]);
      for (std::size_t i = 0; i < N; ++i) V.data_[i] /= norm;
      R.data_[0] = norm;
    }
    else {
      this->dot(V, V, R);
      double G[blocksize * blocksize], U[blocksize * blocksize], Uinv[blocksize * blocksize];
      for (unsigned i = 0; i < blocksize * blocksize; ++i) G[i] = static_cast<double>(R.data_[i]);
      if (!trl_oracle::cholesky_upper(G, blocksize, U)) throw std::runtime_error("Cholesky factorization failed in orthonormalize");
      trl_oracle::inverse_upper(U, blocksize, Uinv);
      for (unsigned i = 0; i < blocksize * blocksize; ++i) R.data_[i] = static_cast<ScalarT>(Uinv[i]);

      auto Vtemp0 = Vtemp->block_view(0);
      V.mult(R, Vtemp0);
      V.copy_from(Vtemp0);

      for (unsigned i = 0; i < blocksize * blocksize; ++i) R.data_[i] = static_cast<ScalarT>(U[i]);
    }
  }

  std::size_t size() const { return N; }

  BlockMultivector create_multivector(std::size_t rows, std::size_t cols) const { return BlockMultivector(rows, cols); }

  BlockMatrix create_blockmatrix(std::size_t block_rows, std::size_t block_cols) const { return BlockMatrix(block_rows, block_cols); }

  // evp_base.hh:79-154
  virtual std::size_t solve_small_dense(const BlockMatrix& B, BlockMatrixBlockView beta, std::size_t nev)
  {
    const auto n_total = B.block_rows() * blocksize;

    std::vector<double> dense(n_total * n_total);
    for (std::size_t i = 0; i < B.block_rows(); ++i)
      for (std::size_t j = 0; j < B.block_cols(); ++j) {
        auto block = B.block_view(i, j);
        for (unsigned int bi = 0; bi < blocksize; ++bi)
          for (unsigned int bj = 0; bj < blocksize; ++bj) dense[(i * blocksize + bi) * n_total + j * blocksize + bj] = block.data_[bi * blocksize + bj];
      }

    std::vector<double> evals(n_total), evecs(n_total * n_total);
    if (!trl_oracle::symmetric_eigen(n_total, dense.data(), evals.data(), evecs.data())) throw std::runtime_error("Eigendecomposition failed");

    // evp_base.hh:101-103 — order by decreasing magnitude
    std::vector<unsigned int> indices(n_total);
    std::iota(indices.begin(), indices.end(), 0);
    std::sort(indices.begin(), indices.end(), [&](const auto& i, const auto& j) { return std::abs(evals[i]) > std::abs(evals[j]); });

    eigenvalues.resize(n_total);
    for (std::size_t i = 0; i < n_total; ++i) eigenvalues[i] = static_cast<Scalar>(evals[indices[i]]);

    if (!eigenvectors) eigenvectors = std::make_unique<BlockMatrix>(B.block_rows(), B.block_cols());
    for (std::size_t i = 0; i < B.block_rows(); ++i)
      for (std::size_t j = 0; j < B.block_cols(); ++j) {
        auto block = eigenvectors->block_view(i, j);
        for (unsigned int bi = 0; bi < blocksize; ++bi)
          for (unsigned int bj = 0; bj < blocksize; ++bj)
            block.data_[bi * blocksize + bj] = static_cast<Scalar>(evecs[(i * blocksize + bi) * n_total + indices[j * blocksize + bj]]);
      }

    // evp_base.hh:124-151 — Ritz estimate ||beta * y_last|| / max(|theta|, eps)
    std::size_t n_converged = 0;
    const std::size_t last_block_row = eigenvectors->block_rows() - 1;
    const ScalarT eps = std::numeric_limits<ScalarT>::epsilon();
    const std::size_t n_check = std::min<std::size_t>(nev, n_total);
    for (std::size_t col_idx = 0; col_idx < n_check; ++col_idx) {
      const std::size_t block_col = col_idx / blocksize;
      const std::size_t col_in_block = col_idx % blocksize;
      auto v_last = eigenvectors->block_view(last_block_row, block_col);
      ScalarT norm_sq = 0.0;
      for (unsigned int i = 0; i < blocksize; ++i) {
        ScalarT sum = 0.0;
        for (unsigned int k = 0; k < blocksize; ++k) sum += beta.data_[i * blocksize + k] * v_last.data_[k * blocksize + col_in_block];
        norm_sq += sum * sum;
      }
      const ScalarT residual_norm = std::sqrt(norm_sq);
      const ScalarT theta = eigenvalues[col_idx];
      const ScalarT denom = std::max(std::abs(theta), eps);
      if (residual_norm / denom < tolerance_) n_converged++;
    }
    return n_converged;
  }

  const std::vector<Scalar>& get_current_eigenvalues() const { return eigenvalues; }

  const BlockMatrix& get_current_eigenvectors() const
  {
    assert(eigenvectors);
    return *eigenvectors;
  }

  std::span<Scalar, blocksize> get_eigenvalues_block(std::size_t block)
  {
    std::span<Scalar, blocksize> ev_block(eigenvalues.data() + block * blocksize, blocksize);
    return ev_block;
  }

  void set_tolerance(Scalar tol) { tolerance_ = tol; }
  Scalar get_tolerance() const { return tolerance_; }

protected:
  std::size_t N;

  std::optional<BlockMultivector> Vtemp;

  std::vector<Scalar> eigenvalues;
  std::unique_ptr<BlockMatrix> eigenvectors;

  Scalar tolerance_ = 1e-8;
};
} // namespace trl::openmp
