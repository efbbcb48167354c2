#pragma once
// Eigenproblem base class of the CUDA backend; the counterpart of trl::openmp::EVPBase
// (impl/openmp/evp_base.hh:13-181). Everything stays on the device:
//  - dot              -> trl_cuda_block_dot (FP64 accumulation)                  (:37)
//  - orthonormalize   -> trl_cuda_cholqr: Cholesky-QR2 by default (one extra pass
//                        restores orthogonality to working precision); passes = 1
//                        reproduces the reference's single CholQR                (:39-71)
//  - solve_small_dense -> trl_cuda_small_eigen: dense FP64 eigensolve of T, sort by
//                        decreasing |theta|, Ritz-estimate count on the device;
//                        only the eigenvalues and the count are copied back      (:79-154)
// The eigenvalues are also kept in host memory because the driver reads them through a
// host std::span (lanczos.hh:129-131).
#include "blockmatrix.hh"
#include "context.hh"
#include "multivector.hh"

#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <random>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <vector>

namespace trl::cuda {

template <class Storage, unsigned int block_size>
class EVPBase {
public:
  using Scalar = double;
  constexpr static auto blocksize = block_size;

  using BlockMultivector = ::trl::cuda::BlockMultivector<Storage, blocksize>;
  using BlockView = typename BlockMultivector::BlockView;
  using BlockMatrix = typename BlockMultivector::BlockMatrix;
  using BlockMatrixBlockView = typename BlockMatrix::BlockView;
  static constexpr int dtype = dtype_of<Storage>::value;

  EVPBase(std::shared_ptr<Context> ctx, std::size_t n)
      : ctx_(std::move(ctx))
      , N(n)
  {
  }

  virtual ~EVPBase() = default;

  virtual void apply(BlockView, BlockView) = 0;

  virtual void dot(BlockView V, BlockView W, BlockMatrixBlockView R) { V.dot(W, R); }

  /// True when dot() is the Euclidean inner product; block Gram-Schmidt strategies use the
  /// multi-block kernels only in that case.
  virtual bool euclidean_dot() const { return true; }

  virtual void orthonormalize(BlockView V, BlockMatrixBlockView R)
  {
    if (!euclidean_dot()) {
      // Cholesky-QR in the eigenproblem's own inner product, as the reference does it
      // (evp_base.hh:39-71: G = dot(V, V), G = U^T U, V <- V U^{-1}, R = U), repeated
      // cholqr_passes times with R accumulated (R <- U_2 U_1)
      if (!mgram_.get()) mgram_ = DeviceBuffer(ctx_, 3 * kCoefBytes);
      double* G = static_cast<double*>(mgram_.get());
      double* Rp = G + blocksize * blocksize;
      double* Rt = Rp + blocksize * blocksize;
      for (int pass = 0; pass < cholqr_passes_; ++pass) {
        this->dot(V, V, BlockMatrixBlockView(ctx_.get(), G));
        const std::size_t blk = sizeof(Storage) * N * blocksize;
        ctx_->prepare({{V.data_, blk, false}, {V.data_, blk, true}, {R.data_, kCoefBytes, true}, {G, 3 * kCoefBytes, true}});
        double* out = pass == 0 ? R.data_ : Rp;
        ctx_->check(trl_cuda_cholqr_gram(ctx_->handle(), dtype, V.data_, static_cast<std::int64_t>(N), blocksize, 1, out, G), "orthonormalize");
        if (pass > 0) {
          ctx_->check(trl_cuda_mb_mult(ctx_->handle(), Rp, R.data_, Rt, blocksize), "orthonormalize");
          ctx_->check(trl_cuda_mb_copy(ctx_->handle(), R.data_, Rt, blocksize, 0), "orthonormalize");
        }
      }
      gram_block_ = nullptr;
      return;
    }
    // The Gram matrix V^T V is reused when the reorthogonalisation that just ran on this
    // very block formed it (and no other operation ran since).
    const bool reuse = gram_block_ == V.data_ && gram_seq_ == ctx_->seq();
    gram_block_ = nullptr;
    const std::size_t blk = sizeof(Storage) * N * blocksize;
    ctx_->prepare({{V.data_, blk, false}, {V.data_, blk, true}, {R.data_, kCoefBytes, true}});
    const double* G0 = reuse ? static_cast<const double*>(gram_.get()) : nullptr;
    ctx_->check(trl_cuda_cholqr_gram(ctx_->handle(), dtype, V.data_, static_cast<std::int64_t>(N), blocksize, cholqr_passes_, R.data_, G0), "orthonormalize");
  }

  std::size_t size() const { return N; }

  BlockMultivector create_multivector(std::size_t rows, std::size_t cols) const { return BlockMultivector(ctx_, rows, cols); }

  BlockMatrix create_blockmatrix(std::size_t block_rows, std::size_t block_cols) const { return BlockMatrix(ctx_, block_rows, block_cols); }

  virtual std::size_t solve_small_dense(const BlockMatrix& B, BlockMatrixBlockView beta, std::size_t nev)
  {
    const std::size_t nblk = B.block_rows();
    const std::size_t n_total = nblk * blocksize;
    if (!eigenvectors || eigenvectors->block_rows() != nblk) {
      eigenvectors = std::make_unique<BlockMatrix>(ctx_, nblk, nblk);
      evals_dev_ = DeviceBuffer(ctx_, sizeof(double) * n_total);
    }
    ctx_->prepare({{B.data(), kCoefBytes * B.block_rows() * B.block_cols(), false},
                   {beta.data_, kCoefBytes, false},
                   {eigenvectors->data(), kCoefBytes * nblk * nblk, true},
                   {evals_dev_.get(), sizeof(double) * n_total, true}});
    eigenvalues.resize(n_total);
    int nconv = 0;
    if (full_eigenvectors_) {
      ctx_->check(trl_cuda_small_eigen(ctx_->handle(), B.data(), static_cast<int>(nblk), blocksize, beta.data_, static_cast<int>(nev), tolerance_,
                                       static_cast<double*>(evals_dev_.get()), eigenvectors->data(), eigenvalues.data(), &nconv),
                  "solve_small_dense");
    }
    else {
      // the driver reads the eigenvectors of the kept blocks only (lanczos.hh:105-131)
      const std::size_t kvec = std::min(n_total, std::max((nev / blocksize + 1) * blocksize, min_eigenvectors_));
      ctx_->check(trl_cuda_small_eigen_partial(ctx_->handle(), B.data(), static_cast<int>(nblk), blocksize, beta.data_, static_cast<int>(nev), tolerance_,
                                               static_cast<int>(kvec), static_cast<double*>(evals_dev_.get()), eigenvectors->data(), eigenvalues.data(), &nconv),
                  "solve_small_dense");
#ifdef TRL_DEBUG_TRACE
      debug_compare_small(B, beta, nev, kvec, nconv);
#endif
    }
    return static_cast<std::size_t>(nconv);
  }

#ifdef TRL_DEBUG_TRACE
  /// Debug builds with TRL_DUMP_SMALL=<dir>: every projected problem is solved again by the
  /// full eigensolver; when the kept eigenvectors disagree (per column, up to sign) the
  /// matrix, beta and both results are written to <dir>.
  void debug_compare_small(const BlockMatrix& B, BlockMatrixBlockView beta, std::size_t nev, std::size_t kvec, int nconv)
  {
    static const char* dir = std::getenv("TRL_DUMP_SMALL");
    static int call = 0;
    if (!dir) return;
    ++call;
    const std::size_t nblk = B.block_rows(), N = nblk * blocksize, NN = N * N;
    DeviceBuffer Yf(ctx_, sizeof(double) * NN), ev(ctx_, sizeof(double) * N);
    std::vector<double> evh(N), yp(NN), yf(NN), Th(NN), bh(blocksize * blocksize);
    int nc2 = 0;
    ctx_->check(trl_cuda_small_eigen(ctx_->handle(), B.data(), static_cast<int>(nblk), blocksize, beta.data_, static_cast<int>(nev), tolerance_,
                                     static_cast<double*>(ev.get()), static_cast<double*>(Yf.get()), evh.data(), &nc2), "debug");
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), yp.data(), eigenvectors->data(), sizeof(double) * NN, TRL_D2H), "debug");
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), yf.data(), Yf.get(), sizeof(double) * NN, TRL_D2H), "debug");
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), Th.data(), B.data(), sizeof(double) * NN, TRL_D2H), "debug");
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), bh.data(), beta.data_, sizeof(double) * blocksize * blocksize, TRL_D2H), "debug");
    auto at = [&](const std::vector<double>& Y, std::size_t r, std::size_t c) { // block layout
      return Y[((r / blocksize) * nblk + c / blocksize) * blocksize * blocksize + (r % blocksize) * blocksize + c % blocksize];
    };
    double worst_ev = 0.0, worst_vec = 0.0;
    std::size_t worst_col = 0;
    for (std::size_t c = 0; c < N; ++c) worst_ev = std::max(worst_ev, std::abs(evh[c] - eigenvalues[c]));
    for (std::size_t c = 0; c < kvec; ++c) {
      double dp = 0.0, dm = 0.0;
      for (std::size_t r = 0; r < N; ++r) {
        dp = std::max(dp, std::abs(at(yp, r, c) - at(yf, r, c)));
        dm = std::max(dm, std::abs(at(yp, r, c) + at(yf, r, c)));
      }
      if (std::min(dp, dm) > worst_vec) {
        worst_vec = std::min(dp, dm);
        worst_col = c;
      }
    }
    std::fprintf(stderr, "small %d N %zu nconv %d/%d ev_diff %.3e vec_diff %.3e col %zu top %.12f %.12f\n", call, N, nconv, nc2, worst_ev, worst_vec, worst_col,
                 eigenvalues[0], eigenvalues[1]);
    static const double dump_above = std::getenv("TRL_DUMP_ABOVE") ? std::atof(std::getenv("TRL_DUMP_ABOVE")) : 1e300;
    static int dumped = 0;
    if (worst_vec > 1e-6 || nconv != nc2 || (std::abs(eigenvalues[0]) > dump_above && dumped++ < 2) || (call >= 1 && std::getenv("TRL_DUMP_ALL"))) {
      const std::string base = std::string(dir) + "/small_" + std::to_string(call);
      if (FILE* f = std::fopen((base + ".bin").c_str(), "wb")) {
        const std::int64_t hdr[4] = {static_cast<std::int64_t>(nblk), blocksize, static_cast<std::int64_t>(kvec), static_cast<std::int64_t>(nev)};
        std::fwrite(hdr, sizeof hdr, 1, f);
        std::fwrite(Th.data(), sizeof(double), NN, f);
        std::fwrite(bh.data(), sizeof(double), bh.size(), f);
        std::fwrite(eigenvalues.data(), sizeof(double), N, f);
        std::fwrite(yp.data(), sizeof(double), NN, f);
        std::fwrite(evh.data(), sizeof(double), N, f);
        std::fwrite(yf.data(), sizeof(double), NN, f);
        std::fclose(f);
      }
    }
  }
#endif

  const std::vector<Scalar>& get_current_eigenvalues() const { return eigenvalues; }

  const BlockMatrix& get_current_eigenvectors() const
  {
    assert(eigenvectors);
    return *eigenvectors;
  }

  std::span<Scalar, blocksize> get_eigenvalues_block(std::size_t block) { return std::span<Scalar, blocksize>(eigenvalues.data() + block * blocksize, blocksize); }

  void set_tolerance(Scalar tol) { tolerance_ = tol; }
  Scalar get_tolerance() const { return tolerance_; }

  // ---- backend extensions --------------------------------------------------------------

  /// Number of Cholesky-QR passes in orthonormalize (2 = CholQR2, 1 = reference CholQR).
  void set_cholqr_passes(int p) { cholqr_passes_ = p; }

  /// true: every eigenvector of the projected problem (cuSOLVER syevd), as the reference's
  /// dense solver computes; false (default): those of the kept blocks only
  /// (trl_cuda_small_eigen_partial), all the driver reads.
  void set_full_eigenvectors(bool on) { full_eigenvectors_ = on; }
  /// Eigenvectors the partial solve forms at least (a caller that forms more Ritz vectors
  /// from the last projected problem than the restart keeps).
  void set_min_eigenvectors(std::size_t k) { min_eigenvectors_ = k; }
  int cholqr_passes() const { return cholqr_passes_; }

  /// Classical Gram-Schmidt of w against the `count` contiguous blocks starting at V0
  /// (trl_cuda_project_out; mode TRL_CGS_ONE / TRL_CGS_TWO / TRL_CGS_IFNEEDED). Keeps the
  /// Gram matrix of the result for the orthonormalize() that follows.
  void project_out(BlockView V0, unsigned int count, BlockView w, int mode, double eta = 0.70710678118654752)
  {
    if (count == 0) return;
    if (!gram_.get()) gram_ = DeviceBuffer(ctx_, sizeof(double) * blocksize * blocksize);
    const std::size_t blk = sizeof(Storage) * N * blocksize;
    ctx_->prepare({{V0.data_, blk * count, false}, {w.data_, blk, false}, {w.data_, blk, true}});
    ctx_->check(trl_cuda_project_out(ctx_->handle(), dtype, V0.data_, static_cast<int>(count), w.data_, static_cast<std::int64_t>(N), blocksize, mode, eta,
                                     static_cast<double*>(gram_.get())),
                "project_out");
    gram_block_ = w.data_;
    gram_seq_ = ctx_->seq();
  }

  /// Partial reorthogonalisation of w against the `count` contiguous blocks starting at V0
  /// (trl_cuda_project_out_sketch): projects only when the random sketch S of those blocks
  /// shows a loss of orthogonality above set_partial_threshold() (default 1e-12). S is kept
  /// here: extended by the blocks added since the last call, rebuilt when the basis changed
  /// (a restart rotates it into the other multivector, or count went down). The sketch
  /// assumes the basis is append-only between those events: a caller that rewrites blocks
  /// already sketched in place (same V0, count not decreasing) calls reset_sketch() first.
  /// The reference driver never does; its restarts swap V and W. With
  /// set_partial_pairs (the default) a step whose test fired also projects the next step:
  /// projected alone, a step leaves the loss of its unprojected predecessor to return two
  /// steps later through the recurrence's B term.
  void project_out_sketch(BlockView V0, unsigned int count, BlockView w, double eta = 0.70710678118654752)
  {
    if (count == 0) return;
    if (!gram_.get()) gram_ = DeviceBuffer(ctx_, sizeof(double) * blocksize * blocksize);
    if (!sketch_.get()) sketch_ = DeviceBuffer(ctx_, sizeof(Storage) * N * blocksize);
    if (!sketch_pair_.get()) {
      sketch_pair_ = DeviceBuffer(ctx_, sizeof(int));
      ctx_->flush();
      ctx_->check(trl_cuda_memset_zero(ctx_->handle(), sketch_pair_.get(), sizeof(int)), "sketch pair state");
    }
    const std::size_t blk = sizeof(Storage) * N * blocksize;
    constexpr std::size_t bb = blocksize * blocksize;
    if (count > sketch_coef_blocks_) { // coefficients G_j, entries N(0, 1/bs), one fixed sequence
      const std::size_t want = std::max<std::size_t>(2 * count, 64);
      std::vector<double> g(want * bb);
      std::mt19937_64 rng(0x5eed5eedULL);
      std::normal_distribution<double> dist(0.0, 1.0 / std::sqrt(static_cast<double>(blocksize)));
      for (auto& x : g) x = dist(rng);
      sketch_coef_ = DeviceBuffer(ctx_, sizeof(double) * g.size());
      ctx_->flush();
      ctx_->check(trl_cuda_memcpy(ctx_->handle(), sketch_coef_.get(), g.data(), sizeof(double) * g.size(), TRL_H2D), "sketch coefficients");
      sketch_coef_blocks_ = want;
    }
    ctx_->prepare({{V0.data_, blk * count, false}, {w.data_, blk, false}, {w.data_, blk, true}, {sketch_.get(), blk, true}});
    const auto h = ctx_->handle();
    const double* coef = static_cast<const double*>(sketch_coef_.get());
    if (V0.data_ != sketch_v0_ || count < sketch_count_) {
      ctx_->check(trl_cuda_block_rotate(h, dtype, V0.data_, static_cast<int>(count), coef, 1, 1, sketch_.get(), static_cast<std::int64_t>(N), blocksize), "sketch");
    }
    else {
      for (std::size_t j = sketch_count_; j < count; ++j)
        ctx_->check(trl_cuda_bv_mult(h, dtype, TRL_MULT_ADD, static_cast<const Storage*>(V0.data_) + j * N * blocksize, coef + j * bb, sketch_.get(),
                                     static_cast<std::int64_t>(N), blocksize),
                    "sketch");
    }
    sketch_v0_ = V0.data_;
    sketch_count_ = count;
    ctx_->check(trl_cuda_project_out_sketch(h, dtype, V0.data_, static_cast<int>(count), w.data_, static_cast<std::int64_t>(N), blocksize, sketch_.get(), partial_threshold_,
                                            eta, static_cast<double*>(gram_.get()), partial_pairs_ ? static_cast<int*>(sketch_pair_.get()) : nullptr),
                "project_out_sketch");
    gram_block_ = w.data_;
    gram_seq_ = ctx_->seq();
  }

  /// FP32 storage resolves orthogonality to ~1e-7 only: its threshold is at least 1e-6.
  void set_partial_threshold(double t) { partial_threshold_ = sizeof(Storage) < 8 ? std::max(t, 1e-6) : t; }
  double partial_threshold() const { return partial_threshold_; }
  void set_partial_pairs(bool on) { partial_pairs_ = on; }
  bool partial_pairs() const { return partial_pairs_; }
  /// Forget the partial reorthogonalisation's sketch and its pending pair: the next
  /// project_out_sketch rebuilds S from the blocks it is given.
  void reset_sketch()
  {
    sketch_v0_ = nullptr;
    sketch_count_ = 0;
    if (sketch_pair_.get()) ctx_->check(trl_cuda_memset_zero(ctx_->handle(), sketch_pair_.get(), sizeof(int)), "sketch pair state");
  }

  Context& context() const { return *ctx_; }
  const std::shared_ptr<Context>& shared_context() const { return ctx_; }
  const double* device_eigenvalues() const { return static_cast<const double*>(evals_dev_.get()); }

protected:
  static constexpr std::size_t kCoefBytes = sizeof(double) * blocksize * blocksize;

  std::shared_ptr<Context> ctx_;
  std::size_t N;

  std::vector<Scalar> eigenvalues;
  std::unique_ptr<BlockMatrix> eigenvectors;
  DeviceBuffer evals_dev_;
  DeviceBuffer gram_;                  // Gram matrix of the last reorthogonalised block
  DeviceBuffer mgram_;                 // non-Euclidean orthonormalize: Gram, pass factor, product
  const Storage* gram_block_ = nullptr; // ... which block it belongs to
  std::uint64_t gram_seq_ = 0;         // ... and the operation sequence number it was made at

  Scalar tolerance_ = 1e-8;
  int cholqr_passes_ = 2;
  bool full_eigenvectors_ = false;
  std::size_t min_eigenvectors_ = 0;
  // partial reorthogonalisation: the sketch of the basis and its coefficients
  double partial_threshold_ = sizeof(Storage) < 8 ? 1e-6 : 1e-12;
  bool partial_pairs_ = true;
  DeviceBuffer sketch_, sketch_coef_, sketch_pair_;
  std::size_t sketch_coef_blocks_ = 0;
  const Storage* sketch_v0_ = nullptr;
  std::size_t sketch_count_ = 0;
};

} // namespace trl::cuda
