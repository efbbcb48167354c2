// The reference's own backend-generic test bodies (tests/test_lanczos_convergence.hh,
// tests/test_lanczos_extend.hh, tests/helpers.hh) instantiated on the CUDA backend, with the
// same cases as the reference's OpenMP test programs (tests/openmp/test_lanczos_convergence.cc
// :17-78 and tests/openmp/test_lanczos_extend.cc:12-47): the diagonal operator
// diag[i] = (i+1)^2 (tests/openmp/diagonal.hh:19) and the 1-D Dirichlet Laplacian
// (tests/openmp/laplace.hh:19-31), N = 128, block sizes 1, 2, 4, 8, FP64, tolerance 1e-8.
// Both operators are given to the backend as CSR matrices, so these tests also exercise the
// SpMM kernel. With the argument "fp32" the convergence bodies run on the FP32-storage
// backend with tolerance 1e-5 (the reference has no single-precision test; its extend test
// uses absolute FP64-level thresholds and is run in FP64 only).
//
// Exit status: number of failed cases (as the reference's programs).
#include "test_lanczos_convergence.hh"
#include "test_lanczos_extend.hh"

#include <trl/impl/cuda/csrevp.hh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iostream>
#include <memory>
#include <random>
#include <string>
#include <vector>

namespace {

using trl::cuda::Context;

template <class Storage, unsigned bs>
std::shared_ptr<trl::cuda::CSREVP<Storage, bs>> make_csr_evp(const std::shared_ptr<Context>& ctx, std::size_t n, bool laplace)
{
  std::vector<std::int32_t> rowptr(n + 1), col;
  std::vector<double> val;
  for (std::size_t i = 0; i < n; ++i) {
    rowptr[i] = static_cast<std::int32_t>(col.size());
    if (laplace && i > 0) {
      col.push_back(static_cast<std::int32_t>(i - 1));
      val.push_back(-1.0);
    }
    col.push_back(static_cast<std::int32_t>(i));
    val.push_back(laplace ? 2.0 : static_cast<double>((i + 1) * (i + 1)));
    if (laplace && i + 1 < n) {
      col.push_back(static_cast<std::int32_t>(i + 1));
      val.push_back(-1.0);
    }
  }
  rowptr[n] = static_cast<std::int32_t>(col.size());
  trl::cuda::DeviceCSR<Storage> A(ctx, static_cast<std::int64_t>(n), static_cast<std::int64_t>(col.size()), rowptr.data(), col.data(), val.data());
  return std::make_shared<trl::cuda::CSREVP<Storage, bs>>(ctx, std::move(A));
}

// Test shim of the backend (the CUDA counterpart of tests/openmp/test_helper.hh and
// tests/sycl/test_helper.hh): default-seeded std::mt19937 + normal_distribution, host copies.
template <trl::Eigenproblem EVP>
class CUDATestHelper {
public:
  using Storage = typename EVP::BlockMultivector::StorageType;
  using BlockView = typename EVP::BlockMultivector::BlockView;
  using MBV = typename EVP::BlockMultivector::BlockMatrix::BlockView;

  explicit CUDATestHelper(std::shared_ptr<Context> ctx)
      : ctx_(std::move(ctx))
  {
  }

  void set_random(BlockView V)
  {
    std::vector<Storage> host(V.rows() * V.cols());
    std::generate(host.begin(), host.end(), [&]() { return static_cast<Storage>(dist(rng)); });
    ctx_->flush();
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), V.data_, host.data(), sizeof(Storage) * host.size(), TRL_H2D), "set_random");
    ctx_->sync();
  }

  double norm(BlockView V)
  {
    std::vector<Storage> host(V.rows() * V.cols());
    ctx_->flush();
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), host.data(), V.data_, sizeof(Storage) * host.size(), TRL_D2H), "norm");
    double s = 0.0;
    for (auto x : host) s += static_cast<double>(x) * static_cast<double>(x);
    return std::sqrt(s);
  }

  std::vector<double> to_host_data(MBV B)
  {
    std::vector<double> host(EVP::blocksize * EVP::blocksize);
    ctx_->flush();
    ctx_->check(trl_cuda_memcpy(ctx_->handle(), host.data(), B.data_, sizeof(double) * host.size(), TRL_D2H), "to_host_data");
    return host;
  }

  std::vector<double> to_host_data(const std::vector<double>& data) { return data; }

  void sync() { ctx_->sync(); }

private:
  std::shared_ptr<Context> ctx_;
  std::mt19937 rng;
  std::normal_distribution<double> dist;
};

template <class Storage, unsigned bs>
bool convergence_case(const std::shared_ptr<Context>& ctx, bool laplace, double tol)
{
  std::cout << "\n[" << (laplace ? "Laplace 1D" : "Diagonal") << " Test: bs=" << bs << "]\n";
  const unsigned N = 128, nev = 16;
  auto evp = make_csr_evp<Storage, bs>(ctx, N, laplace);
  CUDATestHelper<trl::cuda::CSREVP<Storage, bs>> helper(ctx);
  std::vector<double> exact(nev);
  const double pi = std::acos(-1.0);
  for (unsigned i = 0; i < nev; ++i) exact[i] = laplace ? 2.0 - 2.0 * std::cos((N - i) * pi / (N + 1)) : static_cast<double>((N - i) * (N - i));
  return test_lanczos_convergence(evp, helper, exact, tol);
}

template <class Storage, unsigned bs>
bool extend_case(const std::shared_ptr<Context>& ctx, double tol)
{
  auto evp = make_csr_evp<Storage, bs>(ctx, 128, false);
  CUDATestHelper<trl::cuda::CSREVP<Storage, bs>> helper(ctx);
  return test_lanczos_extend(evp, helper, tol, true);
}

template <class Storage>
int run_all(double tol, bool with_extend)
{
  auto ctx = Context::create(0);
  int failed = 0;
  std::cout << "--- Diagonal Eigenvalue Problem ---\n";
  failed += !convergence_case<Storage, 1>(ctx, false, tol);
  failed += !convergence_case<Storage, 2>(ctx, false, tol);
  failed += !convergence_case<Storage, 4>(ctx, false, tol);
  failed += !convergence_case<Storage, 8>(ctx, false, tol);
  std::cout << "\n--- Laplace 1D Eigenvalue Problem ---\n";
  failed += !convergence_case<Storage, 1>(ctx, true, tol);
  failed += !convergence_case<Storage, 2>(ctx, true, tol);
  failed += !convergence_case<Storage, 4>(ctx, true, tol);
  failed += !convergence_case<Storage, 8>(ctx, true, tol);
  if (with_extend) {
    // absolute thresholds on ||A V - V T|| with ||A|| = 128^2: meaningful in FP64 only
    std::cout << "\n--- Lanczos relation (extend) ---\n";
    failed += !extend_case<Storage, 1>(ctx, tol);
    failed += !extend_case<Storage, 2>(ctx, tol);
    failed += !extend_case<Storage, 4>(ctx, tol);
    failed += !extend_case<Storage, 8>(ctx, tol);
  }
  std::cout << "\nTests completed: " << (failed == 0 ? "ALL PASSED" : std::to_string(failed) + " FAILED") << "\n";
  return failed;
}

} // namespace

int main(int argc, char** argv)
{
  try {
    if (argc > 1 && std::strcmp(argv[1], "fp32") == 0) return run_all<float>(1e-5, false);
    return run_all<double>(1e-8, true);
  }
  catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 100;
  }
}
