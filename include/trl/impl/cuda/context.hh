#pragma once
// trl::cuda — B200 (sm_100a) backend for trl's block Lanczos solver.
//
// Context: owns the C-ABI handle (include/trl_cuda.h: one CUDA stream + device workspace),
// turns non-zero ABI status codes into the exception types the reference throws
// (std::invalid_argument, std::runtime_error with the reference's messages,
// impl/openmp/evp_base.hh:55,96), and batches the restart rotation.
//
// Rotation batching. The thick restart (lanczos.hh:105-114) issues, for every kept block j,
// W_j.set_zero() followed by m calls V_i.mult_add(Y_ij, W_j): k*m passes that each re-read
// one basis block. The context records set_zero / mult_add calls instead of launching
// them; the next operation of any other kind flushes the record. When the record is
// exactly "W_j = sum_i V_i Y_ij for consecutive basis blocks V_i, consecutive W_j and one
// block matrix Y", it is issued as one trl_cuda_block_rotate (one pass over V); otherwise
// the calls are replayed one by one in their original order. Results are identical up to
// floating-point summation order.
#include "trl_cuda.h"

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace trl::cuda {

template <class T>
struct dtype_of;
template <>
struct dtype_of<double> {
  static constexpr int value = TRL_F64;
};
template <>
struct dtype_of<float> {
  static constexpr int value = TRL_F32;
};

class Context {
public:
  explicit Context(int device = 0, void* stream = nullptr)
  {
    const int st = trl_cuda_create(&h_, device, stream);
    if (st != TRL_OK) throw std::runtime_error(std::string("trl::cuda: cannot create context: ") + trl_cuda_status_string(st));
  }
  /// Borrows an existing handle (not destroyed with the context).
  explicit Context(trl_cuda_handle borrowed)
      : h_(borrowed)
      , owns_(false)
  {
    if (!h_) throw std::invalid_argument("trl::cuda: null handle");
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  ~Context()
  {
    try {
      flush();
    }
    catch (...) {
    }
    if (owns_) trl_cuda_destroy(h_);
  }

  static std::shared_ptr<Context> create(int device = 0, void* stream = nullptr) { return std::make_shared<Context>(device, stream); }
  static std::shared_ptr<Context> borrow(trl_cuda_handle h) { return std::make_shared<Context>(h); }

  trl_cuda_handle handle() const { return h_; }

  /// Throws for a non-zero ABI status (exception types follow the reference backends).
  void check(int status, const char* what = nullptr) const
  {
    if (status == TRL_OK) return;
    std::string msg = trl_cuda_last_error(h_);
    if (msg.empty()) msg = trl_cuda_status_string(status);
    if (what) msg = std::string(what) + ": " + msg;
    switch (status) {
    case TRL_EINVAL:
    case TRL_ENOTSUP: throw std::invalid_argument(msg);
    case TRL_ECHOLESKY: throw std::runtime_error("Cholesky factorization failed in orthonormalize");
    case TRL_EEIGEN: throw std::runtime_error("Eigendecomposition failed");
    default: throw std::runtime_error(msg);
    }
  }

  /// Issues pending work and waits for the stream; reports device-side breakdowns.
  void sync()
  {
    flush();
    check(trl_cuda_synchronize(h_), "synchronize");
  }

  // ---- recorded (lazy) block-vector operations ---------------------------------------
  struct Op {
    int kind; // 0 = zero(out), 1 = out += in * coef
    int dtype;
    int bs;
    std::int64_t n;
    const void* in;
    const double* coef;
    void* out;
  };

  /// Enables or disables rotation batching (enabled by default).
  void set_batching(bool on)
  {
    flush();
    batching_ = on;
  }
  bool batching() const { return batching_; }

  void record_zero(int dtype, int bs, std::int64_t n, void* out)
  {
    if (!batching_) {
      check(trl_cuda_bv_zero(h_, dtype, out, n, bs), "set_zero");
      return;
    }
    push({0, dtype, bs, n, nullptr, nullptr, out});
  }

  void record_mult_add(int dtype, int bs, std::int64_t n, const void* in, const double* coef, void* out)
  {
    if (!batching_) {
      check(trl_cuda_bv_mult(h_, dtype, TRL_MULT_ADD, in, coef, out, n, bs), "mult_add");
      return;
    }
    push({1, dtype, bs, n, in, coef, out});
  }

  /// Operation sequence number: advances with every backend operation (each one flushes or
  /// records). Lets a result computed by one operation be reused by the next one only if
  /// nothing ran in between.
  std::uint64_t seq() const { return seq_; }

  /// Executes every recorded operation (fused when the pattern allows).
  void flush()
  {
    ++seq_;
    if (pending_.empty()) return;
    std::vector<Op> ops;
    ops.swap(pending_);
    if (try_rotation(ops)) return;
    for (const auto& op : ops) {
      if (op.kind == 0) check(trl_cuda_bv_zero(h_, op.dtype, op.out, op.n, op.bs), "set_zero");
      else check(trl_cuda_bv_mult(h_, op.dtype, TRL_MULT_ADD, op.in, op.coef, op.out, op.n, op.bs), "mult_add");
    }
  }

  /// Number of fused rotations issued so far (diagnostics).
  std::uint64_t fused_rotations() const { return fused_; }

private:
  trl_cuda_handle h_ = nullptr;
  bool owns_ = true;
  bool batching_ = true;
  std::vector<Op> pending_;
  std::uint64_t fused_ = 0;
  std::uint64_t seq_ = 0;

  void push(const Op& op)
  {
    ++seq_;
    if (!pending_.empty()) {
      const Op& f = pending_.front();
      if (f.dtype != op.dtype || f.bs != op.bs || f.n != op.n) flush();
    }
    pending_.push_back(op);
  }

  bool try_rotation(const std::vector<Op>& ops)
  {
    const Op& f = ops.front();
    if (f.kind != 0) return false;
    const std::size_t es = f.dtype == TRL_F64 ? sizeof(double) : sizeof(float);
    const std::ptrdiff_t blk_bytes = static_cast<std::ptrdiff_t>(f.n) * f.bs * static_cast<std::ptrdiff_t>(es);
    const std::ptrdiff_t bb = static_cast<std::ptrdiff_t>(f.bs) * f.bs;
    // groups: [zero(out_j), madd(in_i, coef_ij, out_j) for i < m]
    std::size_t pos = 0;
    int k = 0, m = -1;
    const char* in0 = nullptr;
    const double* c00 = nullptr;
    char* out0 = nullptr;
    std::ptrdiff_t ldc = -1;
    while (pos < ops.size()) {
      const Op& z = ops[pos];
      if (z.kind != 0) return false;
      char* outj = static_cast<char*>(z.out);
      if (k == 0) out0 = outj;
      else if (outj != out0 + k * blk_bytes) return false;
      ++pos;
      int i = 0;
      while (pos < ops.size() && ops[pos].kind == 1) {
        const Op& a = ops[pos];
        if (a.out != z.out) return false;
        const char* ini = static_cast<const char*>(a.in);
        if (k == 0 && i == 0) {
          in0 = ini;
          c00 = a.coef;
        }
        if (ini != in0 + i * blk_bytes) return false;
        const std::ptrdiff_t coff = a.coef - c00; // in doubles
        if (k == 0 && i == 1) {
          if (coff <= 0 || coff % bb != 0) return false;
          ldc = coff / bb;
        }
        if (i > 0 && ldc < 0) return false;
        const std::ptrdiff_t expect = (static_cast<std::ptrdiff_t>(i) * (ldc < 0 ? 0 : ldc) + k) * bb;
        if (coff != expect) return false;
        ++i;
        ++pos;
      }
      if (m < 0) m = i;
      else if (i != m) return false;
      ++k;
    }
    if (m <= 0) return false;
    if (ldc < 0) ldc = k; // a single input block: any ldc >= k addresses the same blocks
    if (ldc < k) return false;
    // the rotation reads V and writes W: they must not overlap
    const char* in_end = in0 + m * blk_bytes;
    const char* out_end = out0 + k * blk_bytes;
    if (out0 < in_end && in0 < out_end) return false;
    check(trl_cuda_block_rotate(h_, f.dtype, in0, m, c00, static_cast<int>(ldc), k, out0, f.n, f.bs), "rotation");
    ++fused_;
    return true;
  }
};

/// RAII device allocation owned through a Context.
class DeviceBuffer {
public:
  DeviceBuffer() = default;
  DeviceBuffer(std::shared_ptr<Context> ctx, std::size_t bytes)
      : ctx_(std::move(ctx))
      , bytes_(bytes)
  {
    ctx_->check(trl_cuda_malloc(ctx_->handle(), &ptr_, bytes), "allocation");
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
  {
    if (this != &o) {
      release();
      swap(o);
    }
    return *this;
  }
  ~DeviceBuffer() { release(); }

  void* get() const { return ptr_; }
  std::size_t bytes() const { return bytes_; }
  Context* context() const { return ctx_.get(); }
  const std::shared_ptr<Context>& shared_context() const { return ctx_; }

private:
  std::shared_ptr<Context> ctx_;
  void* ptr_ = nullptr;
  std::size_t bytes_ = 0;

  void swap(DeviceBuffer& o) noexcept
  {
    std::swap(ctx_, o.ctx_);
    std::swap(ptr_, o.ptr_);
    std::swap(bytes_, o.bytes_);
  }
  void release() noexcept
  {
    if (ptr_ && ctx_) {
      try {
        ctx_->flush(); // recorded operations may still name this buffer
      }
      catch (...) {
      }
      trl_cuda_free(ctx_->handle(), ptr_);
    }
    ptr_ = nullptr;
    bytes_ = 0;
  }
};

} // namespace trl::cuda
