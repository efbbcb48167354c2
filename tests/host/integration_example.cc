// The documented C++ usage: the reference's BlockLanczos over the CUDA backend types, the
// M-inner-product problem and a shared prepared operator. Compiled with -fsyntax-only by
// tests/test_host_logic.py so that the documented API cannot drift.
#include <trl/eigensolvers/lanczos.hh>
#include <trl/impl/cuda/csrevp.hh>
#include <trl/impl/cuda/reorthogonalization.hh>
#include <cstdint>
#include <vector>
int main()
{
  std::int64_t n = 4, nnz = 4;
  std::vector<std::int32_t> rp{0, 1, 2, 3, 4}, ci{0, 1, 2, 3};
  std::vector<double> vals{1, 2, 3, 4}, x0(n * 8);
  const std::int32_t* rowptr = rp.data(); const std::int32_t* colind = ci.data(); const double* values = vals.data(); const double* host_x0 = x0.data();
  auto ctx = trl::cuda::Context::create(/*device=*/0);
  trl::cuda::DeviceCSR<double> A(ctx, n, nnz, rowptr, colind, values);
  using EVP = trl::cuda::CSREVP<double, 8>;
  auto evp = std::make_shared<EVP>(ctx, std::move(A));
  trl::EigensolverParams params{.nev = 32, .ncv = 384, .max_restarts = 1000, .tolerance = 1e-10};
  trl::BlockLanczos<EVP, trl::cuda::BlockCGSIfNeeded> lanczos(evp, params);
  auto V0 = lanczos.initial_block();
  trl_cuda_memcpy(ctx->handle(), V0.data_, host_x0, n * 8 * sizeof(double), TRL_H2D);
  auto result = lanczos.solve();
  auto evals = evp->get_current_eigenvalues();
  (void)result; (void)evals;
  // the M inner product and a shared prepared operator
  trl::cuda::DeviceCSR<double> K(ctx, n, nnz, rowptr, colind, values), M(ctx, n, nnz, rowptr, colind, values);
  auto op = std::make_shared<const trl::cuda::SellOp>(ctx, K.desc(), 8);
  auto evp2 = std::make_shared<trl::cuda::MInnerCSREVP<double, 8>>(ctx, std::move(K), std::move(M), 1.0, 0.0);
  (void)op; (void)evp2;
  return 0;
}
