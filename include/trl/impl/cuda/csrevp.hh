#pragma once
// Sparse operator eigenproblem on the device: Y = alpha*A*X + beta*X with A in full-storage
// CSR (int32 indices). The CUDA counterpart of the reference's CSREVP examples
// (examples/openmp/csrevp.hh:19-48, examples/sycl/csrevp.hh:159-187). The shift turns the
// smallest eigenvalues of A into the largest-magnitude ones of sigma*I - A, which the
// |theta|-descending ordering of solve_small_dense (evp_base.hh:103) selects.
//
// Values are stored in the multivector's Storage type: FP64 for the FP64 backend, FP32 for
// the mixed-precision backend (whose SpMM runs in FP32 with FP32 accumulation).
#include "evp_base.hh"

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <type_traits>
#include <vector>

namespace trl::cuda {

/// Device CSR matrix with values of type V. Owns its arrays when built from host data.
template <class V>
class DeviceCSR {
public:
  DeviceCSR() = default;

  /// Uploads host CSR arrays (values converted to V).
  DeviceCSR(std::shared_ptr<Context> ctx, std::int64_t n, std::int64_t nnz, const std::int32_t* rowptr, const std::int32_t* colind, const double* values)
      : n_(n)
      , nnz_(nnz)
  {
    rowptr_ = DeviceBuffer(ctx, sizeof(std::int32_t) * (n + 1));
    colind_ = DeviceBuffer(ctx, sizeof(std::int32_t) * (nnz > 0 ? nnz : 1));
    values_ = DeviceBuffer(ctx, sizeof(V) * (nnz > 0 ? nnz : 1));
    auto h = ctx->handle();
    ctx->check(trl_cuda_memcpy(h, rowptr_.get(), rowptr, sizeof(std::int32_t) * (n + 1), TRL_H2D), "CSR upload");
    if (nnz > 0) {
      ctx->check(trl_cuda_memcpy(h, colind_.get(), colind, sizeof(std::int32_t) * nnz, TRL_H2D), "CSR upload");
      if constexpr (std::is_same_v<V, double>) {
        ctx->check(trl_cuda_memcpy(h, values_.get(), values, sizeof(double) * nnz, TRL_H2D), "CSR upload");
      }
      else {
        std::vector<V> tmp(values, values + nnz);
        ctx->check(trl_cuda_memcpy(h, values_.get(), tmp.data(), sizeof(V) * nnz, TRL_H2D), "CSR upload");
        ctx->check(trl_cuda_synchronize(h), "CSR upload");
      }
    }
    desc_ = {n_, nnz_, static_cast<const std::int32_t*>(rowptr_.get()), static_cast<const std::int32_t*>(colind_.get()), values_.get(), dtype_of<V>::value};
  }

  /// Wraps device arrays owned by the caller.
  static DeviceCSR wrap(std::int64_t n, std::int64_t nnz, const std::int32_t* rowptr, const std::int32_t* colind, const V* values)
  {
    DeviceCSR c;
    c.n_ = n;
    c.nnz_ = nnz;
    c.desc_ = {n, nnz, rowptr, colind, values, dtype_of<V>::value};
    return c;
  }

  const trl_csr* desc() const { return &desc_; }
  std::int64_t rows() const { return n_; }
  std::int64_t nnz() const { return nnz_; }

private:
  std::int64_t n_ = 0, nnz_ = 0;
  DeviceBuffer rowptr_, colind_, values_;
  trl_csr desc_{};
};

/// The operator prepared for repeated SpMMs with block size bs (trl_cuda_op: a sliced-ELL
/// copy of the CSR matrix, built on the device once). Owns the copy; move-only.
class SellOp {
public:
  SellOp(std::shared_ptr<Context> ctx, const trl_csr* A, int bs)
      : ctx_(std::move(ctx))
  {
    ctx_->flush();
    ctx_->check(trl_cuda_op_create(ctx_->handle(), A, bs, &op_), "operator preparation");
  }
  ~SellOp()
  {
    if (op_) trl_cuda_op_destroy(ctx_->handle(), op_);
  }
  SellOp(const SellOp&) = delete;
  SellOp& operator=(const SellOp&) = delete;

  trl_cuda_op get() const { return op_; }

  /// Y_j = alpha A X_j + beta X_j + gamma W_j, j < nb (a direct ABI call: the caller flushes
  /// the context's recorded operations first when they may touch X, Y or W).
  void spmm(const void* X, void* Y, int nb, double alpha, double beta, double gamma = 0.0, const void* W = nullptr) const
  {
    ctx_->check(trl_cuda_op_spmm(ctx_->handle(), op_, X, Y, nb, alpha, beta, gamma, W), "apply");
  }

private:
  std::shared_ptr<Context> ctx_;
  trl_cuda_op op_ = nullptr;
};

template <class Storage, unsigned int bs>
class CSREVP : public EVPBase<Storage, bs> {
public:
  using Base = EVPBase<Storage, bs>;
  using BlockView = typename Base::BlockView;

  /// op: the operator prepared for this block size (shared with other users of the same
  /// matrix); prepared here when null.
  CSREVP(std::shared_ptr<Context> ctx, DeviceCSR<Storage> A, double alpha = 1.0, double beta = 0.0, std::shared_ptr<const SellOp> op = nullptr)
      : Base(ctx, static_cast<std::size_t>(A.rows()))
      , A_(std::move(A))
      , alpha_(alpha)
      , beta_(beta)
      , op_(op ? std::move(op) : std::make_shared<const SellOp>(ctx, A_.desc(), static_cast<int>(bs)))
  {
  }

  void apply(BlockView X, BlockView Y) override
  {
    const std::size_t blk = sizeof(Storage) * this->N * bs;
    this->ctx_->prepare({{X.data_, blk, false}, {Y.data_, blk, true}});
    op_->spmm(X.data_, Y.data_, 1, alpha_, beta_);
    ++applies_;
  }

  const DeviceCSR<Storage>& matrix() const { return A_; }
  double alpha() const { return alpha_; }
  double beta() const { return beta_; }
  std::uint64_t applies() const { return applies_; }

private:
  DeviceCSR<Storage> A_;
  double alpha_, beta_;
  std::shared_ptr<const SellOp> op_;
  std::uint64_t applies_ = 0;
};

} // namespace trl::cuda

namespace trl::cuda {

/// Eigenproblem with a matrix-weighted inner product: apply = the CSR operator `op`
/// (Y = alpha*op*X + beta*X), dot(V, W) = V^T (M W) with M an SPD CSR matrix, and CholQR in
/// that inner product (EVPBase::orthonormalize goes through dot() when euclidean_dot() is
/// false). The CUDA counterpart of the reference's generalised example
/// (examples/openmp/csrevp.hh:52-109: apply = (A - sigma B)^{-1} B, dot = V^T (B W)), with the
/// operator given explicitly: any operator that is self-adjoint in the M inner product, such
/// as M^{-1} K for K x = lambda M x. The Ritz vectors come out M-orthonormal.
template <class Storage, unsigned int bs>
class MInnerCSREVP : public CSREVP<Storage, bs> {
public:
  using Base = CSREVP<Storage, bs>;
  using BlockView = typename Base::BlockView;
  using BlockMatrixBlockView = typename Base::BlockMatrixBlockView;

  MInnerCSREVP(std::shared_ptr<Context> ctx, DeviceCSR<Storage> op, DeviceCSR<Storage> M, double alpha = 1.0, double beta = 0.0)
      : Base(ctx, std::move(op), alpha, beta)
      , M_(std::move(M))
      , mop_(std::make_shared<const SellOp>(ctx, M_.desc(), static_cast<int>(bs)))
      , MW_(ctx, sizeof(Storage) * this->N * bs)
  {
    if (M_.rows() != static_cast<std::int64_t>(this->N)) throw std::invalid_argument("M must have the operator's size");
  }

  /// R = V^T (M W)                                   (examples/openmp/csrevp.hh:89-97)
  void dot(BlockView V, BlockView W, BlockMatrixBlockView R) override
  {
    const std::size_t blk = sizeof(Storage) * this->N * bs;
    this->ctx_->prepare({{V.data_, blk, false}, {W.data_, blk, false}, {MW_.get(), blk, true}, {R.data_, sizeof(double) * bs * bs, true}});
    mop_->spmm(W.data_, MW_.get(), 1, 1.0, 0.0);
    this->ctx_->check(trl_cuda_block_dot(this->ctx_->handle(), Base::dtype, V.data_, 1, MW_.get(), static_cast<std::int64_t>(this->N), bs, R.data_), "dot");
  }

  bool euclidean_dot() const override { return false; }

  const DeviceCSR<Storage>& mass() const { return M_; }

private:
  DeviceCSR<Storage> M_;
  std::shared_ptr<const SellOp> mop_;
  DeviceBuffer MW_;
};

} // namespace trl::cuda
