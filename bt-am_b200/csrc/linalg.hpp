// Small dense host linear algebra of the solvers: the least-squares step of
// N-GMRES (a symmetric positive semi-definite Gram system of at most 16
// unknowns).
#pragma once

#include <algorithm>
#include <cmath>

namespace btam {

// H beta = b in the least-squares sense with the minimum-norm solution, for
// a symmetric positive semi-definite H (n x n, row-major, n <= 16): cyclic
// Jacobi rotations to H = V diag(l) V^T, then beta = V diag(1/l) V^T b over
// the eigenvalues above 2.2e-16 times the largest (those below are dropped,
// as an SVD solve with a machine-precision cutoff drops them).  b is
// overwritten with beta; H is left as it is.
inline void lsq_sym(int n, const double *H, double *b) {
  constexpr int N = 16;
  double A[N][N], V[N][N];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      A[i][j] = H[i * n + j];
      V[i][j] = i == j ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i) {
      diag += A[i][i] * A[i][i];
      for (int j = i + 1; j < n; ++j) off += A[i][j] * A[i][j];
    }
    if (!(off > 1e-32 * diag)) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        if (A[p][q] == 0.0) continue;
        const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A J
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- J^T A
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {  // V <- V J
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  double lmax = 0.0;
  for (int i = 0; i < n; ++i) lmax = std::max(lmax, std::fabs(A[i][i]));
  double y[N] = {0.0};
  for (int k = 0; k < n; ++k) {
    if (!(std::fabs(A[k][k]) > 2.220446049250313e-16 * lmax)) continue;
    double vb = 0.0;
    for (int i = 0; i < n; ++i) vb += V[i][k] * b[i];
    for (int i = 0; i < n; ++i) y[i] += V[i][k] * vb / A[k][k];
  }
  for (int i = 0; i < n; ++i) b[i] = y[i];
}

}  // namespace btam
