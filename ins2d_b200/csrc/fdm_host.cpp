// Generalized eigen-decompositions of the 1D factors of the pressure matrix
// A = -(diag(hy) (x) TX + TY (x) diag(hx)) (the separable form of
// A = M Om^-1 G, operator_divergence.m:208), for the fast-diagonalization
// preconditioner of the device PCG.
#include "fdm_host.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>

namespace ins2d {

namespace {

// A (symmetric, row-major) = Q T Q' with T tridiagonal (diagonal d, off
// diagonal e[i] = T(i, i+1), e[n-1] = 0); Q row-major.  Householder
// reflections H = I - 2 v v' applied to the trailing block column by column.
void householder_tridiagonal(int n, std::vector<double> &A, std::vector<double> &Q, std::vector<double> &d,
                             std::vector<double> &e) {
  Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
  std::vector<double> v(n), p(n), q(n);
  for (int k = 0; k + 2 < n; ++k) {
    // v = x - alpha e1 for x = A(k+1:n, k)
    double nx2 = 0.0;
    for (int i = k + 1; i < n; ++i) nx2 += A[(size_t)i * n + k] * A[(size_t)i * n + k];
    const double nx = std::sqrt(nx2);
    double tail2 = nx2 - A[(size_t)(k + 1) * n + k] * A[(size_t)(k + 1) * n + k];
    if (nx == 0.0 || tail2 <= 1e-300 * std::max(1.0, nx2)) continue;  // already tridiagonal in this column
    const double x0 = A[(size_t)(k + 1) * n + k];
    const double alpha = x0 >= 0.0 ? -nx : nx;
    for (int i = 0; i < n; ++i) v[i] = 0.0;
    for (int i = k + 1; i < n; ++i) v[i] = A[(size_t)i * n + k];
    v[k + 1] -= alpha;
    double nv2 = 0.0;
    for (int i = k + 1; i < n; ++i) nv2 += v[i] * v[i];
    const double inv = 1.0 / std::sqrt(nv2);
    for (int i = k + 1; i < n; ++i) v[i] *= inv;
    // trailing block B = A(k+1:, k+1:): B <- H B H = B - 2 v q' - 2 q v',
    // p = B v, q = p - (v'p) v
    for (int i = k + 1; i < n; ++i) {
      double s = 0.0;
      const double *row = &A[(size_t)i * n];
      for (int j = k + 1; j < n; ++j) s += row[j] * v[j];
      p[i] = s;
    }
    double K = 0.0;
    for (int i = k + 1; i < n; ++i) K += v[i] * p[i];
    for (int i = k + 1; i < n; ++i) q[i] = p[i] - K * v[i];
    for (int i = k + 1; i < n; ++i) {
      double *row = &A[(size_t)i * n];
      for (int j = k + 1; j < n; ++j) row[j] -= 2.0 * (v[i] * q[j] + q[i] * v[j]);
    }
    A[(size_t)(k + 1) * n + k] = alpha;
    A[(size_t)k * n + k + 1] = alpha;
    for (int i = k + 2; i < n; ++i) A[(size_t)i * n + k] = A[(size_t)k * n + i] = 0.0;
    // Q <- Q H
    for (int i = 0; i < n; ++i) {
      double *row = &Q[(size_t)i * n];
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += row[j] * v[j];
      s *= 2.0;
      for (int j = k + 1; j < n; ++j) row[j] -= s * v[j];
    }
  }
  d.assign(n, 0.0);
  e.assign(n, 0.0);
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i];
  for (int i = 0; i + 1 < n; ++i) e[i] = A[(size_t)i * n + i + 1];
}

// Implicit QL iteration on the tridiagonal (d, e) with the eigenvectors
// accumulated into Z (row-major, columns = vectors).
void tridiagonal_ql(int n, std::vector<double> &d, std::vector<double> &e, std::vector<double> &Z) {
  const double eps = std::numeric_limits<double>::epsilon();
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= eps * dd) break;
      }
      if (m == l) break;
      if (++iter > 60) throw std::runtime_error("eigen-decomposition did not converge");
      // shift: eigenvalue of the leading 2x2 block of rows l, l+1 nearer d[l]
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        double f = s * e[i];
        const double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // underflow: the block splits here
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; ++k) {
          double *row = &Z[(size_t)k * n];
          f = row[i + 1];
          row[i + 1] = s * row[i] + c * f;
          row[i] = c * row[i] - s * f;
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
}

}  // namespace

void sym_eig(int n, std::vector<double> &A, std::vector<double> &V, std::vector<double> &w) {
  std::vector<double> Q, d, e;
  householder_tridiagonal(n, A, Q, d, e);
  tridiagonal_ql(n, d, e, Q);
  // ascending order
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] < d[b]; });
  V.assign((size_t)n * n, 0.0);
  w.assign(n, 0.0);
  for (int a = 0; a < n; ++a) {
    w[a] = d[ord[a]];
    for (int i = 0; i < n; ++i) V[(size_t)i * n + a] = Q[(size_t)i * n + ord[a]];
  }
}

FdmHost1D fdm_1d(const Table &T, const std::vector<double> &h) {
  const int n = T.nrows;
  if (T.ncols != n || (int)h.size() != n) throw std::runtime_error("fdm: factor is not square");
  // S = diag(h)^-1/2 T diag(h)^-1/2, symmetrised against rounding
  std::vector<double> S((size_t)n * n, 0.0), rs(n);
  for (int i = 0; i < n; ++i) rs[i] = 1.0 / std::sqrt(h[i]);
  for (int i = 0; i < n; ++i)
    for (const auto &kv : T.T.rows[i]) S[(size_t)i * n + kv.first] += kv.second * rs[i] * rs[kv.first];
  for (int i = 0; i < n; ++i)
    for (int k = i + 1; k < n; ++k) {
      const double a = 0.5 * (S[(size_t)i * n + k] + S[(size_t)k * n + i]);
      S[(size_t)i * n + k] = S[(size_t)k * n + i] = a;
    }
  FdmHost1D F;
  F.n = n;
  std::vector<double> W;
  sym_eig(n, S, W, F.lam);
  F.Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int a = 0; a < n; ++a) F.Q[(size_t)i * n + a] = W[(size_t)i * n + a] * rs[i];
  // eigenvalues of a semidefinite factor: clip rounding below zero
  const double top = n ? std::fabs(F.lam[n - 1]) : 0.0;
  for (double &l : F.lam)
    if (l < 0.0 && l > -1e-12 * top) l = 0.0;
  return F;
}

}  // namespace ins2d
