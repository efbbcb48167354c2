#pragma once
// Small dense blocks in device memory: BlockMatrix (a grid of bs x bs FP64 blocks) and its
// non-owning block view. Layout and semantics follow the reference OpenMP types
// (impl/openmp/blockmatrix.hh:19-65, impl/openmp/matrixblockview.hh:16-77): block (i,j) is
// row-major at data + (i*block_cols + j)*bs*bs, zero-initialised on construction. Entries
// are FP64 in every precision mode: the projected problem, the Cholesky factors and the
// Gram blocks are always kept in FP64.
#include "context.hh"

#include <cstddef>
#include <memory>
#include <span>
#include <stdexcept>

namespace trl::cuda {

template <unsigned int block_size>
class BlockMatrixBlockView {
public:
  using EntryType = double;

  BlockMatrixBlockView(Context* ctx, double* data)
      : ctx_(ctx)
      , data_(data)
  {
  }

  /// A = B                                   (matrixblockview.hh:30-33)
  void copy_from(BlockMatrixBlockView other)
  {
    ctx_->prepare({{other.data_, kBytes, false}, {data_, kBytes, true}});
    ctx_->check(trl_cuda_mb_copy(ctx_->handle(), data_, other.data_, block_size, 0), "copy_from");
  }

  /// A = B^T                                 (matrixblockview.hh:39-43)
  void copy_from_transpose(BlockMatrixBlockView other)
  {
    ctx_->prepare({{other.data_, kBytes, false}, {data_, kBytes, true}});
    ctx_->check(trl_cuda_mb_copy(ctx_->handle(), data_, other.data_, block_size, 1), "copy_from_transpose");
  }

  /// A = 0                                   (matrixblockview.hh:49)
  void set_zero()
  {
    ctx_->prepare({{data_, kBytes, true}});
    ctx_->check(trl_cuda_mb_zero(ctx_->handle(), data_, block_size), "set_zero");
  }

  /// C = A B                                 (matrixblockview.hh:55-64)
  void mult(BlockMatrixBlockView B, BlockMatrixBlockView C) const
  {
    ctx_->prepare({{data_, kBytes, false}, {B.data_, kBytes, false}, {C.data_, kBytes, true}});
    ctx_->check(trl_cuda_mb_mult(ctx_->handle(), data_, B.data_, C.data_, block_size), "mult");
  }

  /// A(i,i) = values[i] from host memory; off-diagonal entries unchanged  (matrixblockview.hh:71-74)
  void set_diagonal(std::span<double> values)
  {
    if (values.size() < block_size) throw std::invalid_argument("set_diagonal: need blocksize values");
    ctx_->prepare({{data_, kBytes, false}, {data_, kBytes, true}});
    ctx_->check(trl_cuda_mb_set_diagonal(ctx_->handle(), data_, values.data(), block_size), "set_diagonal");
  }

  Context* ctx_;
  double* data_; // device pointer

private:
  static constexpr std::size_t kBytes = sizeof(double) * block_size * block_size;
};

template <unsigned int block_size>
class BlockMatrix {
public:
  using BlockView = BlockMatrixBlockView<block_size>;

  BlockMatrix(std::shared_ptr<Context> ctx, std::size_t brows, std::size_t bcols)
      : block_rows_(brows)
      , block_cols_(bcols)
      , buf_(ctx, sizeof(double) * brows * bcols * block_size * block_size)
  {
    ctx->check(trl_cuda_memset_zero(ctx->handle(), buf_.get(), buf_.bytes()), "BlockMatrix zero");
  }

  BlockMatrix(const BlockMatrix&) = delete;
  BlockMatrix& operator=(const BlockMatrix&) = delete;
  BlockMatrix(BlockMatrix&&) noexcept = default;
  BlockMatrix& operator=(BlockMatrix&&) noexcept = default;

  std::size_t block_rows() const { return block_rows_; }
  std::size_t block_cols() const { return block_cols_; }

  BlockView block_view(std::size_t block_row, std::size_t block_col) const
  {
    if (block_row >= block_rows_ || block_col >= block_cols_) throw std::out_of_range("BlockMatrix::block_view index out of range");
    return BlockView(buf_.context(), data() + (block_row * block_cols_ + block_col) * block_size * block_size);
  }

  double* data() const { return static_cast<double*>(buf_.get()); }
  Context* context() const { return buf_.context(); }

private:
  std::size_t block_rows_;
  std::size_t block_cols_;
  DeviceBuffer buf_;
};

} // namespace trl::cuda
