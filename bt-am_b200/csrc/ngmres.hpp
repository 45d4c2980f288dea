// N-GMRES for the three stretches of the bulk stretch relaxation: host code
// over a residual callback (point.cu calls it with the device residual; the
// CPU tests call it with synthetic residuals).
#pragma once

#include <cmath>
#include <functional>

#include "../../include/btam.h"
#include "linalg.hpp"

namespace btam {

// The reference's configured solver for the stretch equations: SNES type
// "ngmres" with m = 3 and line search "cp" (main-BT-AM.cpp:64-67, the
// options of the "minV_dF_" solver that Mechanical-Relaxation-bulk.cpp:296-341
// sets up).  N-GMRES (Oosterlee and Washio, SIAM J. Sci. Comput. 21 (2000)
// 1670-1690) as PETSc's SNESNGMRES forms it with its defaults: each
// iteration takes a residual step x^M = x - lambda F(x) whose lambda comes
// from the critical-point line search (one secant step on F(x - lambda F)
// . F from lambda = 0 and 1), then the combination x^A of x^M and the last
// m iterates that minimises the linearised residual norm; x^A is kept when
// |F(x^A)| < 2 min|F| and either 0.1 |x^A - x^M| < min_i |x^A - x_i| or
// sqrt|F(x)| < 0.9 sqrt(min|F|), else x^M; the subspace restarts after two
// consecutive iterations with (0.1 |x^A - x^M| > min_i |x^A - x_i| and
// sqrt|F(x^A)| > 0.9 sqrt(min|F|)) or |F(x^A)| > 2 min|F|.  Three residual
// evaluations per iteration.  Returns the status as relax_stretch's loop.
inline double ngmres_norm3(const double y[3]) {
  return std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
}

inline int ngmres_stretch(const std::function<int(const double *, double *)> &residual, int m,
                          double atol, double rtol, int max_iter, double X[3], double Y[3],
                          double n0, int &it, int &status) {
  constexpr double gammaA = 2.0, gammaC = 2.0, epsilonB = 0.1, deltaB = 0.9;
  constexpr int restart_it = 2;
  if (m < 1) m = 1;
  if (m > 3) m = 3;  // the stretch has three unknowns
  double Xs[3][3], Fs[3][3], Q[3][3];  // subspace: iterates, residuals, Gram
  auto dot = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  auto put = [&](int iv, const double *x, const double *f) {
    for (int a = 0; a < 3; ++a) {
      Xs[iv][a] = x[a];
      Fs[iv][a] = f[a];
    }
  };
  double fnorm = ngmres_norm3(Y), fminnorm = fnorm;
  put(0, X, Y);
  int k_restart = 1, l = 1, ivec = 0, restart_count = 0;
  for (int k = 1; k <= max_iter; ++k) {
    // x^M: the critical-point line search along -F from x
    double XM[3], FM[3], W[3];
    const double fty0 = dot(Y, Y);
    double lambda = 1.0;
    if (std::fabs(fty0) >= 1e-15 * fnorm) {
      for (int a = 0; a < 3; ++a) W[a] = X[a] - lambda * Y[a];
      int st = residual(W, FM);
      if (st != BTAM_OK) return st;
      const double fty = dot(FM, Y);
      double sl = (fty - fty0) / lambda;  // secant slope from lambda_old = 0
      if (sl > 0.0) sl = -sl;
      // already at a critical point to the line search's relative tolerance
      // (1e-8): keep lambda = 1
      if (sl != 0.0 && !(std::fabs(fty) / std::fabs(fty0) < 1e-8)) {
        double lu = lambda - fty / sl;
        if (lu < 1e-12) lu = lambda + fty / sl;
        if (std::isfinite(lu) && lu <= 1e8) lambda = lu;
      }
    }
    for (int a = 0; a < 3; ++a) XM[a] = X[a] - lambda * Y[a];
    int st = residual(XM, FM);
    if (st != BTAM_OK) return st;
    const double fMnorm = ngmres_norm3(FM);
    // x^A: the combination minimising |(1 - sum beta) F^M + sum beta F_i|
    double xi[3], beta[3], H[3][3];
    for (int i = 0; i < l; ++i) {
      xi[i] = dot(FM, Fs[i]);
      Q[i][ivec] = Q[ivec][i] = dot(Fs[ivec], Fs[i]);
    }
    const double nu = fMnorm * fMnorm;
    for (int i = 0; i < l; ++i) beta[i] = nu - xi[i];
    for (int j = 0; j < l; ++j)
      for (int i = 0; i < l; ++i) H[i][j] = Q[i][j] - xi[i] - xi[j] + nu;
    if (l == 1) {
      beta[0] = H[0][0] != 0.0 ? beta[0] / H[0][0] : 0.0;
    } else {
      double Hf[9];
      for (int i = 0; i < l; ++i)
        for (int j = 0; j < l; ++j) Hf[i * l + j] = H[i][j];
      lsq_sym(l, Hf, beta);
    }
    double alph = 0.0;
    for (int i = 0; i < l; ++i) alph += beta[i];
    double XA[3], FA[3];
    for (int a = 0; a < 3; ++a) {
      XA[a] = (1.0 - alph) * XM[a];
      for (int i = 0; i < l; ++i) XA[a] += beta[i] * Xs[i][a];
    }
    if ((st = residual(XA, FA)) != BTAM_OK) return st;
    if (fminnorm > fMnorm) fminnorm = fMnorm;
    const double fAnorm = ngmres_norm3(FA);
    double D[3], dnorm, dminnorm = -1.0;
    for (int a = 0; a < 3; ++a) D[a] = XA[a] - XM[a];
    dnorm = ngmres_norm3(D);
    for (int i = 0; i < l; ++i) {
      for (int a = 0; a < 3; ++a) D[a] = Xs[i][a] - XA[a];
      const double dc = ngmres_norm3(D);
      if (dc < dminnorm || dminnorm < 0.0) dminnorm = dc;
    }
    // selection
    bool selA = fAnorm < gammaA * fminnorm;
    if (!(epsilonB * dnorm < dminnorm || std::sqrt(fnorm) < deltaB * std::sqrt(fminnorm)))
      selA = false;
    if (selA) {
      for (int a = 0; a < 3; ++a) {
        X[a] = XA[a];
        Y[a] = FA[a];
      }
      fnorm = fAnorm;
    } else {
      for (int a = 0; a < 3; ++a) {
        X[a] = XM[a];
        Y[a] = FM[a];
      }
      fnorm = fMnorm;
    }
    // restart
    bool rs = false;
    if (epsilonB * dnorm > dminnorm && std::sqrt(fAnorm) > deltaB * std::sqrt(fminnorm)) rs = true;
    if (fAnorm > gammaC * fminnorm) rs = true;
    restart_count = rs ? restart_count + 1 : 0;
    ivec = k_restart % m;
    if (restart_count >= restart_it) {
      restart_count = 0;
      k_restart = 1;
      l = 1;
      ivec = 0;
      put(0, XM, FM);
    } else {
      if (l < m) ++l;
      ++k_restart;
      if (fminnorm > fnorm) fminnorm = fnorm;
      put(ivec, X, Y);
    }
    it = k;
    if (fnorm <= atol || fnorm <= rtol * n0) {
      status = 1;
      return BTAM_OK;
    }
    if (!std::isfinite(fnorm)) return BTAM_ERR_NONFINITE;
  }
  return BTAM_OK;
}

}  // namespace btam
