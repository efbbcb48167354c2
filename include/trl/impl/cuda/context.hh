#pragma once
// trl::cuda — B200 (sm_100a) backend for trl's block Lanczos solver.
//
// Context: owns the C-ABI handle (include/trl_cuda.h: one CUDA stream + device workspace),
// turns non-zero ABI status codes into the exception types the reference throws
// (std::invalid_argument, std::runtime_error with the reference's messages,
// impl/openmp/evp_base.hh:55,96), and defers two call patterns of the driver so that they
// can be fused.
//
// Rotation batching. The thick restart (lanczos.hh:105-114) issues, for every kept block j,
// W_j.set_zero() followed by m calls V_i.mult_add(Y_ij, W_j): k*m passes that each re-read
// one basis block. The context records set_zero / mult_add calls instead of launching
// them; the next operation of any other kind flushes the record. When the record is
// exactly "W_j = sum_i V_i Y_ij for consecutive basis blocks V_i, consecutive W_j and one
// block matrix Y", it is issued as one trl_cuda_block_rotate (one pass over V); otherwise
// the calls are replayed one by one in their original order. Results are identical up to
// floating-point summation order.
//
// Three-term fusion. Every block Lanczos step (lanczos.hh:243-262; after a restart
// :167-183) reduces W = A V_i against its neighbours before the full reorthogonalisation:
// W0 = V_{i-1} beta^T, W -= W0, T_ii = V_i^T W, W0 = V_i T_ii, W -= W0 (W0 a temporary
// block). The context records these mult / mult_transpose / -= / dot calls and issues them
// when the next operation of another kind arrives, in order, with every "product into a
// temporary, then subtract the temporary" pair issued as one W -= X M kernel (three block
// passes instead of five). The arithmetic is that of the calls one by one; only the
// temporary's write is deferred. (Folding the step into the Gram-Schmidt projection that
// follows would save more, but a single projection pass over the unreduced W loses
// orthogonality geometrically: the step is the first of two effective passes.)
//
// Deferred writes. The temporary's last product (W0 = V_i T_ii) is written only if a later
// operation reads W0, writes part of it, or writes V_i or T_ii first; it is dropped when an
// operation overwrites all of W0 (the driver's next step does). Operations state what they
// read and write through prepare(); flush() writes everything. Code that calls the C ABI
// directly on this context's handle must call flush() first.
#include "trl_cuda.h"

#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace trl::cuda {

/// Device allocation failed (TRL_ENOMEM); a std::runtime_error, as the reference's errors.
struct out_of_device_memory : std::runtime_error {
  using std::runtime_error::runtime_error;
};
/// A bounded device-side wait gave up (TRL_ETIMEOUT).
struct device_timeout : std::runtime_error {
  using std::runtime_error::runtime_error;
};

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
    case TRL_ENOMEM: throw out_of_device_memory(msg);
    case TRL_ETIMEOUT: throw device_timeout(msg);
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

  /// Memory an operation reads or writes (device addresses; for deferred writes).
  struct Access {
    const void* ptr;
    std::size_t bytes;
    bool write;
  };

  /// Enables or disables rotation batching and three-term fusion (enabled by default).
  void set_batching(bool on)
  {
    flush();
    batching_ = on;
  }
  bool batching() const { return batching_; }

  void record_zero(int dtype, int bs, std::int64_t n, void* out)
  {
    const std::size_t blk = block_bytes(dtype, bs, n);
    replay_terms();
    guard({{out, blk, true}});
    if (!batching_) {
      ++seq_;
      flush_rotation();
      check(trl_cuda_bv_zero(h_, dtype, out, n, bs), "set_zero");
      return;
    }
    push({0, dtype, bs, n, nullptr, nullptr, out});
  }

  void record_mult_add(int dtype, int bs, std::int64_t n, const void* in, const double* coef, void* out)
  {
    const std::size_t blk = block_bytes(dtype, bs, n);
    replay_terms();
    guard({{in, blk, false}, {coef, coef_bytes(bs), false}, {out, blk, false}, {out, blk, true}});
    if (!batching_) {
      ++seq_;
      flush_rotation();
      check(trl_cuda_bv_mult(h_, dtype, TRL_MULT_ADD, in, coef, out, n, bs), "mult_add");
      return;
    }
    push({1, dtype, bs, n, in, coef, out});
  }

  // ---- three-term calls (recorded for fusion) -----------------------------------------
  // A record holds calls on one block w and one temporary t in the driver's grammar
  // (mult into t, then w -= t; dots of basis blocks with w). A call that does not continue
  // the record first issues it; a call that cannot start one runs at once.

  /// t = x m (transpose: t = x m^T)                      BlockView::mult / mult_transpose
  void record_mult(int dtype, int bs, std::int64_t n, const void* x, const double* m, void* t, bool transpose)
  {
    ++seq_;
    const std::size_t blk = block_bytes(dtype, bs, n);
    flush_rotation();
    const TermOp op{transpose ? kMultT : kMult, dtype, bs, n, x, m, t, nullptr, nullptr};
    const bool starts = batching_ && !overlaps(x, blk, t, blk);
    const bool continues = starts && !terms_.empty() && same_shape(terms_.front(), op) && !is_mult(terms_.back()) && (!term_t_ || term_t_ == t) &&
                           (!term_w_ || (!overlaps(t, blk, term_w_, blk) && !overlaps(x, blk, term_w_, blk)));
    if (!continues) replay_terms();
    guard({{x, blk, false}, {m, coef_bytes(bs), false}, {t, blk, true}});
    if (!starts) {
      run(op);
      return;
    }
    terms_.push_back(op);
    term_t_ = t;
  }

  /// w -= t                                              BlockView::operator-=
  void record_sub(int dtype, int bs, std::int64_t n, void* w, const void* t)
  {
    ++seq_;
    const std::size_t blk = block_bytes(dtype, bs, n);
    flush_rotation();
    const TermOp op{kSub, dtype, bs, n, nullptr, nullptr, const_cast<void*>(t), w, nullptr};
    const bool continues = batching_ && !terms_.empty() && is_mult(terms_.back()) && terms_.back().t == t && same_shape(terms_.front(), op) &&
                           (!term_w_ || term_w_ == w) && !overlaps(w, blk, t, blk) && !overlaps(w, blk, terms_.back().x, blk);
    if (!continues) replay_terms();
    guard({{w, blk, false}, {w, blk, true}, {t, blk, false}});
    if (!continues) {
      run(op);
      return;
    }
    terms_.push_back(op);
    term_w_ = w;
  }

  /// r = x^T w                                           BlockView::dot
  void record_dot(int dtype, int bs, std::int64_t n, const void* x, const void* w, double* r)
  {
    ++seq_;
    const std::size_t blk = block_bytes(dtype, bs, n);
    flush_rotation();
    const TermOp op{kDot, dtype, bs, n, x, nullptr, nullptr, const_cast<void*>(w), r};
    const bool starts = batching_ && !overlaps(x, blk, w, blk);
    const bool continues = starts && !terms_.empty() && same_shape(terms_.front(), op) && !is_mult(terms_.back()) && (!term_w_ || term_w_ == w) &&
                           (!term_t_ || (!overlaps(w, blk, term_t_, blk) && !overlaps(x, blk, term_t_, blk)));
    if (!continues) replay_terms();
    guard({{x, blk, false}, {w, blk, false}, {r, coef_bytes(bs), true}});
    if (!starts) {
      run(op);
      return;
    }
    terms_.push_back(op);
    term_w_ = const_cast<void*>(w);
  }

  /// Before an operation that states the memory it reads and writes: writes or drops the
  /// deferred product as needed and issues every recorded call.
  void prepare(std::initializer_list<Access> acc)
  {
    ++seq_;
    replay_terms();
    flush_rotation();
    guard(acc);
  }

  /// Operation sequence number: advances with every backend operation (each one flushes or
  /// records). Lets a result computed by one operation be reused by the next one only if
  /// nothing ran in between.
  std::uint64_t seq() const { return seq_; }

  /// Executes every recorded and deferred operation (fused when the pattern allows).
  void flush()
  {
    ++seq_;
    replay_terms();
    flush_rotation();
    if (has_deferred_) write_deferred();
  }

  /// Number of fused rotations issued so far (diagnostics).
  std::uint64_t fused_rotations() const { return fused_; }
  /// Number of product/subtract pairs issued as one kernel (diagnostics).
  std::uint64_t fused_pairs() const { return fused_pairs_; }
  /// Number of deferred products that had to be written (diagnostics).
  std::uint64_t deferred_writes() const { return deferred_written_; }

private:
  enum { kMult = 0, kMultT = 1, kSub = 2, kDot = 3 };
  struct TermOp {
    int kind;
    int dtype;
    int bs;
    std::int64_t n;
    const void* x;   // mult / dot: basis block
    const double* m; // mult: coefficient block
    void* t;         // mult: product (temporary); sub: subtrahend
    void* w;         // sub: w -= t; dot: r = x^T w
    double* r;       // dot: result block
  };

  trl_cuda_handle h_ = nullptr;
  bool owns_ = true;
  bool batching_ = true;
  std::vector<Op> pending_;
  std::vector<TermOp> terms_;
  void* term_w_ = nullptr; // the block the recorded three-term calls reduce
  void* term_t_ = nullptr; // their temporary
  TermOp deferred_{};
  bool has_deferred_ = false;
  std::uint64_t fused_ = 0;
  std::uint64_t fused_pairs_ = 0;
  std::uint64_t deferred_written_ = 0;
  std::uint64_t seq_ = 0;

  static std::size_t block_bytes(int dtype, int bs, std::int64_t n)
  {
    return static_cast<std::size_t>(n) * static_cast<std::size_t>(bs) * (dtype == TRL_F64 ? sizeof(double) : sizeof(float));
  }
  static std::size_t coef_bytes(int bs) { return sizeof(double) * static_cast<std::size_t>(bs) * static_cast<std::size_t>(bs); }
  static bool overlaps(const void* a, std::size_t na, const void* b, std::size_t nb)
  {
    const auto pa = reinterpret_cast<std::uintptr_t>(a), pb = reinterpret_cast<std::uintptr_t>(b);
    return na > 0 && nb > 0 && pa < pb + nb && pb < pa + na;
  }
  static bool is_mult(const TermOp& op) { return op.kind == kMult || op.kind == kMultT; }
  static bool same_shape(const TermOp& a, const TermOp& b) { return a.dtype == b.dtype && a.bs == b.bs && a.n == b.n; }

  void run(const TermOp& op)
  {
    switch (op.kind) {
    case kMult: check(trl_cuda_bv_mult(h_, op.dtype, TRL_MULT, op.x, op.m, op.t, op.n, op.bs), "mult"); break;
    case kMultT: check(trl_cuda_bv_mult(h_, op.dtype, TRL_MULT_TRANSPOSE, op.x, op.m, op.t, op.n, op.bs), "mult_transpose"); break;
    case kSub: check(trl_cuda_bv_sub(h_, op.dtype, op.w, op.t, op.n, op.bs), "operator-="); break;
    default: check(trl_cuda_block_dot(h_, op.dtype, op.x, 1, op.w, op.n, op.bs, op.r), "dot"); break;
    }
  }

  /// Issues the recorded three-term calls in order; "t = x m, w -= t" pairs become one
  /// w -= x m kernel and t = x m a deferred write. Each call is first checked against the
  /// deferred product (which may have been made by an earlier pair of the same record).
  void replay_terms()
  {
    if (terms_.empty()) return;
    std::vector<TermOp> ops;
    ops.swap(terms_);
    term_w_ = term_t_ = nullptr;
    for (std::size_t p = 0; p < ops.size(); ++p) {
      const TermOp& op = ops[p];
      const std::size_t blk = block_bytes(op.dtype, op.bs, op.n), cb = coef_bytes(op.bs);
      if (is_mult(op) && p + 1 < ops.size() && ops[p + 1].kind == kSub && ops[p + 1].t == op.t && !overlaps(ops[p + 1].w, blk, op.x, blk) &&
          !overlaps(ops[p + 1].w, blk, op.t, blk)) {
        void* w = ops[p + 1].w;
        if (has_deferred_ && deferred_.t == op.t) has_deferred_ = false; // overwritten by this product
        guard({{op.x, blk, false}, {op.m, cb, false}, {w, blk, false}, {w, blk, true}});
        if (has_deferred_) write_deferred(); // keep one deferred product at a time
        check(trl_cuda_bv_mult(h_, op.dtype, op.kind == kMultT ? TRL_SUBTRACT_TRANSPOSE : TRL_SUBTRACT, op.x, op.m, w, op.n, op.bs), "operator-=");
        deferred_ = op;
        has_deferred_ = true;
        ++fused_pairs_;
        ++p;
        continue;
      }
      switch (op.kind) {
      case kMult:
      case kMultT: guard({{op.x, blk, false}, {op.m, cb, false}, {op.t, blk, true}}); break;
      case kSub: guard({{op.w, blk, false}, {op.w, blk, true}, {op.t, blk, false}}); break;
      default: guard({{op.x, blk, false}, {op.w, blk, false}, {op.r, cb, true}}); break;
      }
      run(op);
    }
  }

  void write_deferred()
  {
    has_deferred_ = false;
    ++deferred_written_;
    run(deferred_);
  }

  /// The deferred product commutes with everything recorded after it; an operation that
  /// reads its output, writes part of it, or writes its inputs needs it written first; one
  /// that overwrites all of its output (and reads none of it) makes it dead.
  void guard(std::initializer_list<Access> acc)
  {
    if (!has_deferred_) return;
    const TermOp& d = deferred_;
    const std::size_t blk = block_bytes(d.dtype, d.bs, d.n), cb = coef_bytes(d.bs);
    bool conflict = false, overwritten = false;
    for (const auto& a : acc) {
      if (a.write && (overlaps(a.ptr, a.bytes, d.x, blk) || overlaps(a.ptr, a.bytes, d.m, cb))) conflict = true;
      if (overlaps(a.ptr, a.bytes, d.t, blk)) {
        if (a.write && a.ptr == d.t && a.bytes >= blk) overwritten = true;
        else conflict = true;
      }
    }
    if (conflict) write_deferred();
    else if (overwritten) has_deferred_ = false;
  }

  void flush_rotation()
  {
    if (pending_.empty()) return;
    std::vector<Op> ops;
    ops.swap(pending_);
    if (try_rotation(ops)) return;
    for (const auto& op : ops) {
      if (op.kind == 0) check(trl_cuda_bv_zero(h_, op.dtype, op.out, op.n, op.bs), "set_zero");
      else check(trl_cuda_bv_mult(h_, op.dtype, TRL_MULT_ADD, op.in, op.coef, op.out, op.n, op.bs), "mult_add");
    }
  }

  void push(const Op& op)
  {
    ++seq_;
    if (!pending_.empty()) {
      const Op& f = pending_.front();
      if (f.dtype != op.dtype || f.bs != op.bs || f.n != op.n) flush_rotation();
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
