// C shim over the solvers' small dense least-squares solve
// (bt-am_b200/csrc/linalg.hpp), built with g++ for the CPU tests.
#include "../../bt-am_b200/csrc/linalg.hpp"

extern "C" {
void lsq_sym_c(int n, const double *H, double *b) { btam::lsq_sym(n, H, b); }
}
