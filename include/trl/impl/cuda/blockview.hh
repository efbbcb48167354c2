#pragma once
// Non-owning view of one n x bs block of a device multivector; the CUDA counterpart of
// trl::openmp::BlockView (impl/openmp/blockview.hh:19-206). Storage is the element type in
// HBM (double, or float for the mixed-precision mode); every small coefficient block is
// FP64 (BlockMatrixBlockView) and every inner product is accumulated in FP64.
#include "blockmatrix.hh"
#include "context.hh"

#include <cstddef>

namespace trl::cuda {

template <class Storage, unsigned int block_size>
class BlockView {
public:
  constexpr static auto blocksize = block_size;
  using EntryType = Storage;
  using MatrixBlockView = BlockMatrixBlockView<block_size>;
  static constexpr int dtype = dtype_of<Storage>::value;

  BlockView(Context* ctx, Storage* data, std::size_t n)
      : data_(data)
      , ctx_(ctx)
      , n_(n)
  {
  }

  std::size_t rows() const { return n_; }
  constexpr std::size_t cols() const { return block_size; }

  /// X = 0 (recorded; see Context)          blockview.hh:31-36
  void set_zero() { ctx_->record_zero(dtype, block_size, static_cast<std::int64_t>(n_), data_); }

  /// X = Y                                   blockview.hh:59-63
  void copy_from(BlockView other)
  {
    ctx_->prepare({{other.data_, bytes(), false}, {data_, bytes(), true}});
    ctx_->check(trl_cuda_bv_copy(ctx_->handle(), dtype, data_, other.data_, static_cast<std::int64_t>(n_), block_size), "copy_from");
  }

  /// X -= Y                                  blockview.hh:69-74
  BlockView& operator-=(BlockView other)
  {
    ctx_->record_sub(dtype, block_size, static_cast<std::int64_t>(n_), data_, other.data_);
    return *this;
  }

  /// other += X W (recorded; see Context)   blockview.hh:81-97
  void mult_add(MatrixBlockView W, BlockView other) { ctx_->record_mult_add(dtype, block_size, static_cast<std::int64_t>(n_), data_, W.data_, other.data_); }

  /// other = X W (recorded; see Context)    blockview.hh:104-119
  void mult(MatrixBlockView W, BlockView other) { ctx_->record_mult(dtype, block_size, static_cast<std::int64_t>(n_), data_, W.data_, other.data_, false); }

  /// other = X W^T (recorded; see Context)  blockview.hh:126-141
  void mult_transpose(MatrixBlockView W, BlockView other) { ctx_->record_mult(dtype, block_size, static_cast<std::int64_t>(n_), data_, W.data_, other.data_, true); }

  /// R = X^T other (FP64, deterministic; recorded, see Context)   blockview.hh:152-182
  void dot(BlockView other, MatrixBlockView R) { ctx_->record_dot(dtype, block_size, static_cast<std::int64_t>(n_), data_, other.data_, R.data_); }

  /// X -= other R                            blockview.hh:189-201
  void subtract_product(BlockView other, MatrixBlockView R)
  {
    ctx_->prepare({{other.data_, bytes(), false}, {R.data_, sizeof(double) * block_size * block_size, false}, {data_, bytes(), false}, {data_, bytes(), true}});
    ctx_->check(trl_cuda_bv_mult(ctx_->handle(), dtype, TRL_SUBTRACT, other.data_, R.data_, data_, static_cast<std::int64_t>(n_), block_size), "subtract_product");
  }

  Storage* data_; // device pointer
  Context* ctx_;

private:
  std::size_t n_;

  std::size_t bytes() const { return sizeof(Storage) * n_ * block_size; }
};

} // namespace trl::cuda
