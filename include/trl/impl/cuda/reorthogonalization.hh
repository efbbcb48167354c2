#pragma once
// Reorthogonalisation strategies for the CUDA backend. They plug into the solver through
// its `Reorth` template parameter (lanczos.hh:22) and satisfy
// trl::ReorthogonalizationStrategy (reorthogonalization.hh:29-32).
//
// BlockCGS2 replaces ModifiedGS (reorthogonalization.hh:12-22). ModifiedGS makes `count`
// rounds of {dot with V_j, subtract V_j C_j}, each re-reading w and one basis block. The
// basis blocks are contiguous in memory ([blocks][n][bs]), so one classical Gram-Schmidt
// pass is a single multi-block inner product C = [V_0..V_{count-1}]^T w followed by a
// single update w -= [V_0..V_{count-1}] C; a second pass ("twice is enough") restores the
// orthogonality that classical Gram-Schmidt loses relative to modified Gram-Schmidt.
// When the eigenproblem's dot() is not the Euclidean product it falls back to two rounds
// of the per-block loop.
#include <concepts>

namespace trl::cuda {

struct BlockCGS2 {
  int passes = 2;

  template <typename EVP, typename BMV>
  void operator()(EVP& evp, BMV& V, unsigned int count, typename BMV::BlockView V_next, typename BMV::BlockMatrix::BlockView tmp) const
  {
    if (count == 0) return;
    if constexpr (requires { evp.project_out(V.block_view(0), count, V_next, 2); }) {
      if (evp.euclidean_dot()) {
        evp.project_out(V.block_view(0), count, V_next, passes);
        return;
      }
    }
    for (int p = 0; p < passes; ++p)
      for (unsigned int j = 0; j < count; ++j) {
        auto Vj = V.block_view(j);
        evp.dot(Vj, V_next, tmp);
        V_next.subtract_product(Vj, tmp);
      }
  }
};

/// One classical Gram-Schmidt pass (no re-orthogonalisation pass).
struct BlockCGS1 : BlockCGS2 {
  BlockCGS1() { passes = 1; }
};

} // namespace trl::cuda
