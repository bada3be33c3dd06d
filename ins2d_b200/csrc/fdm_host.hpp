// Host side of the fast-diagonalization preconditioner (fdm.cu): the
// generalized eigen-decompositions of the 1D factors of the pressure matrix.
#pragma once

#include <vector>

#include "setup.hpp"

namespace ins2d {

// T q = lambda diag(h) q for a symmetric positive semidefinite n x n matrix
// T: Q (row-major, Q[i*n + a] = q_a(i)) with Q' diag(h) Q = I, lam ascending.
struct FdmHost1D {
  int n = 0;
  std::vector<double> Q, lam;
};
FdmHost1D fdm_1d(const Table &T, const std::vector<double> &h);

// Eigen-decomposition of a symmetric n x n matrix A (row-major, destroyed):
// A = V diag(w) V', V row-major (V[i*n + a] = component i of eigenvector a),
// w ascending.  Householder reduction to tridiagonal form, then the implicit
// QL iteration with Wilkinson-type shifts (Bowdler, Martin, Reinsch and
// Wilkinson's algorithm), eigenvectors accumulated.  Throws on no convergence.
void sym_eig(int n, std::vector<double> &A, std::vector<double> &V, std::vector<double> &w);

// largest 1D size for which the context builds the preconditioner (the
// set-up is O(n^3) on the host, the application four dense products)
constexpr int kFdmMaxN = 1024;

}  // namespace ins2d
