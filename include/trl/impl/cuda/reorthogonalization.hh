#pragma once
// Reorthogonalisation strategies for the CUDA backend. They plug into the solver through
// its `Reorth` template parameter (lanczos.hh:22) and satisfy
// trl::ReorthogonalizationStrategy (reorthogonalization.hh:29-32).
//
// They replace ModifiedGS (reorthogonalization.hh:12-22), which makes `count` rounds of
// {dot with V_j, subtract V_j C_j}, each re-reading w and one basis block. The basis blocks
// are contiguous in memory ([blocks][n][bs]), so one classical Gram-Schmidt pass is a
// single multi-block inner product C = [V_0..V_{count-1}]^T w and a single update
// w -= [V_0..V_{count-1}] C (trl_cuda_project_out):
//   BlockCGS1        one pass;
//   BlockCGS2        two passes ("twice is enough");
//   BlockCGSIfNeeded a second pass only when a column kept less than eta of its norm in the
//                    first one (the DGKS criterion), decided on the device. In the Lanczos
//                    recurrence the vector entering the reorthogonalisation is already
//                    orthogonal to the basis up to rounding, so the second pass is rarely
//                    taken and each step reads the basis twice instead of four times.
// The last pass also forms the Gram matrix of the result, which the following
// orthonormalize() reuses. When the eigenproblem's dot() is not the Euclidean product the
// strategies fall back to the per-block loop (passes as above, two for IfNeeded).
#include "trl_cuda.h"

#include <concepts>

namespace trl::cuda {

namespace detail {
template <typename EVP, typename BMV>
void per_block_gram_schmidt(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp, int passes)
{
  for (int p = 0; p < passes; ++p)
    for (unsigned int j = 0; j < count; ++j) {
      auto Vj = V.block_view(j);
      evp.dot(Vj, V_next, tmp);
      V_next.subtract_product(Vj, tmp);
    }
}

template <int Mode, int FallbackPasses, typename EVP, typename BMV>
void classical_gram_schmidt(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp, double eta)
{
  if (count == 0) return;
  if constexpr (requires { evp.project_out(V.block_view(0), count, V_next, Mode, eta); }) {
    if (evp.euclidean_dot()) {
      evp.project_out(V.block_view(0), count, V_next, Mode, eta);
      return;
    }
  }
  per_block_gram_schmidt(evp, V, count, V_next, tmp, FallbackPasses);
}
} // namespace detail

struct BlockCGS1 {
  template <typename EVP, typename BMV>
  void operator()(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp) const
  {
    detail::classical_gram_schmidt<TRL_CGS_ONE, 1>(evp, V, count, V_next, tmp, 0.0);
  }
};

struct BlockCGS2 {
  template <typename EVP, typename BMV>
  void operator()(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp) const
  {
    detail::classical_gram_schmidt<TRL_CGS_TWO, 2>(evp, V, count, V_next, tmp, 0.0);
  }
};

/// Partial reorthogonalisation: the full projection (with the DGKS second pass where
/// needed) only at the steps where a random sketch of the basis shows a loss of
/// orthogonality above the eigenproblem's partial_threshold(); the Lanczos recurrence's own
/// orthogonalisation against the last two blocks (lanczos.hh:240-253) runs every step.
struct BlockCGSPartial {
  double eta = 0.70710678118654752;

  template <typename EVP, typename BMV>
  void operator()(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp) const
  {
    if (count == 0) return;
    if constexpr (requires { evp.project_out_sketch(V.block_view(0), count, V_next, eta); }) {
      if (evp.euclidean_dot()) {
        evp.project_out_sketch(V.block_view(0), count, V_next, eta);
        return;
      }
    }
    detail::per_block_gram_schmidt(evp, V, count, V_next, tmp, 2);
  }
};

struct BlockCGSIfNeeded {
  double eta = 0.70710678118654752; // 1/sqrt(2)

  template <typename EVP, typename BMV>
  void operator()(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp) const
  {
    detail::classical_gram_schmidt<TRL_CGS_IFNEEDED, 2>(evp, V, count, V_next, tmp, eta);
  }
};

} // namespace trl::cuda
