// C shims over the solvers' host pieces (bt-am_b200/csrc/linalg.hpp,
// ngmres.hpp), built with g++ for the CPU tests.
#include "../../bt-am_b200/csrc/linalg.hpp"

extern "C" {
void lsq_sym_c(int n, const double *H, double *b) { btam::lsq_sym(n, H, b); }
}

// The stretch solver's N-GMRES (bt-am_b200/csrc/ngmres.hpp) over a C
// residual callback.
#include "../../bt-am_b200/csrc/ngmres.hpp"

extern "C" {
typedef int (*residual_fn)(const double *x, double *f);
int ngmres3_c(residual_fn res, int m, double atol, double rtol, int max_iter, double *X,
              double *Y, double n0, int *it, int *status) {
  std::function<int(const double *, double *)> r = [res](const double *x, double *f) {
    return res(x, f);
  };
  return btam::ngmres_stretch(r, m, atol, rtol, max_iter, X, Y, n0, *it, *status);
}
}
