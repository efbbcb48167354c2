#pragma once
// Device multivector: `cols/bs` blocks of n x bs, block-major ([blocks][n][bs], block i at
// data + i*n*bs), zero-initialised, move-only — the layout and ownership rules of
// trl::openmp::BlockMultivector (impl/openmp/multivector.hh:19-97). Scalar (the type of the
// projected problem and of tolerances) is double; Storage is the element type in HBM.
#include "blockmatrix.hh"
#include "blockview.hh"
#include "context.hh"

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>

namespace trl::cuda {

template <class Storage, unsigned int block_size>
class BlockMultivector {
public:
  using Scalar = double;
  using StorageType = Storage;
  using BlockView = ::trl::cuda::BlockView<Storage, block_size>;
  using BlockMatrix = ::trl::cuda::BlockMatrix<block_size>;
  using MatrixBlockView = typename BlockMatrix::BlockView;

  static constexpr auto blocksize = block_size;

  BlockMultivector(std::shared_ptr<Context> ctx, std::size_t rows, std::size_t cols)
      : rows_(rows)
      , blocks_(cols / block_size)
  {
    if (cols % block_size != 0) throw std::invalid_argument("Number of columns must be divisible by blocksize");
    buf_ = DeviceBuffer(ctx, sizeof(Storage) * rows * cols);
    ctx->check(trl_cuda_memset_zero(ctx->handle(), buf_.get(), buf_.bytes()), "BlockMultivector zero");
  }

  BlockMultivector(const BlockMultivector&) = delete;
  BlockMultivector& operator=(const BlockMultivector&) = delete;
  BlockMultivector(BlockMultivector&&) noexcept = default;
  BlockMultivector& operator=(BlockMultivector&&) noexcept = default;

  BlockView block_view(std::size_t i) const
  {
    if (i >= blocks_) throw std::out_of_range("Block " + std::to_string(i) + " is out of bounds (number of blocks is " + std::to_string(blocks_) + ")");
    return BlockView(buf_.context(), data() + i * rows_ * block_size, rows_);
  }

  std::size_t blocks() const { return blocks_; }
  std::size_t rows() const { return rows_; }
  Storage* data() const { return static_cast<Storage*>(buf_.get()); }
  Context* context() const { return buf_.context(); }

private:
  std::size_t rows_ = 0;
  std::size_t blocks_ = 0;
  DeviceBuffer buf_;
};

} // namespace trl::cuda
