// TEST INFRASTRUCTURE ONLY — part of the CPU oracle. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py may build, load or run anything under oracle/.
//
// Small dense FP64 linear algebra that the reference obtains from Eigen
// (include/trl/impl/openmp/evp_base.hh:53-60 uses Eigen::LLT and MatrixBase::inverse;
// :95 uses Eigen::SelfAdjointEigenSolver). Eigen is not installed here, so these are
// written from the mathematics:
//   * Cholesky G = L L^T reading the lower triangle, failing on a pivot <= 0 — the
//     failure rule of a standard LL^T factorisation (Golub & Van Loan, Alg. 4.2.1);
//   * inverse of an upper-triangular matrix by back substitution;
//   * symmetric eigensolver: Householder tridiagonalisation (Golub & Van Loan, Alg. 8.3.1)
//     followed by the implicit symmetric QR step with Wilkinson shift (Alg. 8.3.2/8.3.3),
//     eigenvalues returned in ascending order with their eigenvectors as columns, which
//     is the ordering contract of Eigen::SelfAdjointEigenSolver.
// Parity with Eigen itself is unpinned (no reference test pins Eigen's outputs); it is
// pinned end to end by the reference's analytic known-answer tests.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <limits>
#include <numeric>
#include <vector>

namespace trl_oracle {

/// G (b x b, row-major, only the lower triangle is read) = L L^T. On success writes
/// U = L^T (upper triangular, row-major) and returns true; returns false when a pivot
/// is not strictly positive (or NaN).
inline bool cholesky_upper(const double* G, unsigned b, double* U)
{
  std::vector<double> L(static_cast<std::size_t>(b) * b, 0.0);
  for (unsigned j = 0; j < b; ++j) {
    double d = G[j * b + j];
    for (unsigned k = 0; k < j; ++k) d -= L[j * b + k] * L[j * b + k];
    if (!(d > 0.0)) return false;
    const double ljj = std::sqrt(d);
    L[j * b + j] = ljj;
    for (unsigned i = j + 1; i < b; ++i) {
      double s = G[i * b + j];
      for (unsigned k = 0; k < j; ++k) s -= L[i * b + k] * L[j * b + k];
      L[i * b + j] = s / ljj;
    }
  }
  for (unsigned i = 0; i < b; ++i)
    for (unsigned j = 0; j < b; ++j) U[i * b + j] = L[j * b + i];
  return true;
}

/// Inverse of an upper-triangular b x b matrix (row-major) by back substitution.
inline void inverse_upper(const double* U, unsigned b, double* Uinv)
{
  std::fill_n(Uinv, static_cast<std::size_t>(b) * b, 0.0);
  for (unsigned c = 0; c < b; ++c) {
    // solve U x = e_c; x has zeros below row c
    for (int i = static_cast<int>(c); i >= 0; --i) {
      double s = (static_cast<unsigned>(i) == c) ? 1.0 : 0.0;
      for (unsigned k = i + 1; k <= c; ++k) s -= U[i * b + k] * Uinv[k * b + c];
      Uinv[i * b + c] = s / U[i * b + i];
    }
  }
}

/// Symmetric eigendecomposition of the n x n matrix A (row-major; only the lower triangle
/// is read). On return evals[0..n) ascending and evecs (row-major n x n) holds the
/// eigenvector of evals[j] in column j. Returns false if the QR iteration fails to converge.
inline bool symmetric_eigen(std::size_t n, const double* A, double* evals, double* evecs)
{
  if (n == 0) return true;
  // a: working symmetric copy, row-major.
  std::vector<double> a(n * n);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j <= i; ++j) a[i * n + j] = a[j * n + i] = A[i * n + j];

  // ---- Householder tridiagonalisation: Q^T A Q = tridiag(d, e) ----
  std::vector<double> d(n), e(n, 0.0);
  std::vector<std::vector<double>> hv; // Householder vectors (length n, zero-padded)
  std::vector<double> hbeta;
  std::vector<double> p(n), w(n);
  for (std::size_t k = 0; k + 2 < n; ++k) {
    // x = a[k+1:n, k]
    double sigma = 0.0;
    for (std::size_t i = k + 2; i < n; ++i) sigma += a[i * n + k] * a[i * n + k];
    const double x0 = a[(k + 1) * n + k];
    std::vector<double> v(n, 0.0);
    if (sigma == 0.0) {
      hv.push_back(std::move(v));
      hbeta.push_back(0.0);
      continue;
    }
    const double mu = std::sqrt(x0 * x0 + sigma);
    // choose the sign that avoids cancellation: v0 = x0 + sign(x0) * mu
    const double v0 = (x0 >= 0.0) ? x0 + mu : x0 - mu;
    v[k + 1] = 1.0;
    for (std::size_t i = k + 2; i < n; ++i) v[i] = a[i * n + k] / v0;
    double vtv = 0.0;
    for (std::size_t i = k + 1; i < n; ++i) vtv += v[i] * v[i];
    const double beta = 2.0 / vtv;
    // p = beta * A22 v
    for (std::size_t i = k + 1; i < n; ++i) {
      double s = 0.0;
      const double* row = &a[i * n];
      for (std::size_t j = k + 1; j < n; ++j) s += row[j] * v[j];
      p[i] = beta * s;
    }
    double ptv = 0.0;
    for (std::size_t i = k + 1; i < n; ++i) ptv += p[i] * v[i];
    const double coef = 0.5 * beta * ptv;
    for (std::size_t i = k + 1; i < n; ++i) w[i] = p[i] - coef * v[i];
    for (std::size_t i = k + 1; i < n; ++i) {
      double* row = &a[i * n];
      const double vi = v[i], wi = w[i];
      for (std::size_t j = k + 1; j < n; ++j) row[j] -= vi * w[j] + wi * v[j];
    }
    // the reflected column becomes (-sign(x0) mu, 0, ..., 0)
    const double newval = (x0 >= 0.0) ? -mu : mu;
    a[(k + 1) * n + k] = a[k * n + k + 1] = newval;
    for (std::size_t i = k + 2; i < n; ++i) a[i * n + k] = a[k * n + i] = 0.0;
    hv.push_back(std::move(v));
    hbeta.push_back(beta);
  }
  for (std::size_t i = 0; i < n; ++i) d[i] = a[i * n + i];
  for (std::size_t i = 0; i + 1 < n; ++i) e[i] = a[(i + 1) * n + i];

  // zt = Q^T stored row-major, so that row j of zt is column j of Q. Q = H_0 H_1 ... H_{n-3}.
  // Build Q^T = H_{n-3} ... H_0 applied to I from the right: accumulate backwards on Q.
  std::vector<double> q(n * n, 0.0);
  for (std::size_t i = 0; i < n; ++i) q[i * n + i] = 1.0;
  for (std::size_t kk = hv.size(); kk-- > 0;) {
    const auto& v = hv[kk];
    const double beta = hbeta[kk];
    if (beta == 0.0) continue;
    const std::size_t k = kk;
    // Q <- H_k Q, H_k = I - beta v v^T acting on rows k+1..n-1
    for (std::size_t j = k + 1; j < n; ++j) w[j] = 0.0;
    for (std::size_t i = k + 1; i < n; ++i) {
      const double vi = v[i];
      const double* row = &q[i * n];
      for (std::size_t j = k + 1; j < n; ++j) w[j] += vi * row[j];
    }
    for (std::size_t i = k + 1; i < n; ++i) {
      const double f = beta * v[i];
      double* row = &q[i * n];
      for (std::size_t j = k + 1; j < n; ++j) row[j] -= f * w[j];
    }
  }
  std::vector<double> zt(n * n);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j < n; ++j) zt[j * n + i] = q[i * n + j];

  // ---- implicit symmetric QR with Wilkinson shift on (d, e) ----
  const double eps = std::numeric_limits<double>::epsilon();
  std::size_t hi = n - 1;
  int iter_budget = static_cast<int>(60 * n + 100);
  auto rotate_rows = [&](std::size_t r0, std::size_t r1, double c, double s) {
    double* x = &zt[r0 * n];
    double* y = &zt[r1 * n];
    for (std::size_t t = 0; t < n; ++t) {
      const double xv = x[t], yv = y[t];
      x[t] = c * xv - s * yv;
      y[t] = s * xv + c * yv;
    }
  };
  while (hi > 0) {
    // deflate negligible sub-diagonal entries
    for (std::size_t i = 0; i < hi; ++i)
      if (std::abs(e[i]) <= eps * (std::abs(d[i]) + std::abs(d[i + 1]))) e[i] = 0.0;
    while (hi > 0 && e[hi - 1] == 0.0) --hi;
    if (hi == 0) break;
    std::size_t lo = hi - 1;
    while (lo > 0 && e[lo - 1] != 0.0) --lo;
    if (--iter_budget < 0) return false;
    // Wilkinson shift from the trailing 2x2 of the unreduced block [lo, hi]
    const double tdiff = 0.5 * (d[hi - 1] - d[hi]);
    const double eh = e[hi - 1];
    const double denom = tdiff + ((tdiff >= 0.0) ? 1.0 : -1.0) * std::hypot(tdiff, eh);
    const double mu = d[hi] - eh * eh / denom;
    // implicit QR step: chase the bulge from lo to hi
    double x = d[lo] - mu;
    double z = e[lo];
    for (std::size_t k = lo; k < hi; ++k) {
      // Givens (c, s) with [c s; -s c]^T [x; z] = [r; 0]
      double c, s;
      if (z == 0.0) {
        c = 1.0;
        s = 0.0;
      }
      else if (std::abs(z) > std::abs(x)) {
        const double tau = -x / z;
        s = 1.0 / std::sqrt(1.0 + tau * tau);
        c = s * tau;
      }
      else {
        const double tau = -z / x;
        c = 1.0 / std::sqrt(1.0 + tau * tau);
        s = c * tau;
      }
      // apply G^T T G on rows/cols k, k+1 of the tridiagonal matrix
      if (k > lo) e[k - 1] = c * e[k - 1] - s * z;
      const double dk = d[k], dk1 = d[k + 1], ek = e[k];
      const double cc = c * c, ss = s * s, cs = c * s;
      d[k] = cc * dk - 2.0 * cs * ek + ss * dk1;
      d[k + 1] = ss * dk + 2.0 * cs * ek + cc * dk1;
      e[k] = cs * (dk - dk1) + (cc - ss) * ek;
      if (k + 1 < hi) {
        x = e[k];
        z = -s * e[k + 1];
        e[k + 1] = c * e[k + 1];
      }
      rotate_rows(k, k + 1, c, s);
    }
  }

  // ---- sort ascending ----
  std::vector<std::size_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](std::size_t i, std::size_t j) { return d[i] < d[j]; });
  for (std::size_t j = 0; j < n; ++j) {
    evals[j] = d[idx[j]];
    const double* src = &zt[idx[j] * n];
    for (std::size_t i = 0; i < n; ++i) evecs[i * n + j] = src[i];
  }
  return true;
}

} // namespace trl_oracle
