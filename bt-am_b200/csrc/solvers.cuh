// Device kernels of the relaxation and of the hydrogen master equation.
#pragma once

#include <cuda_runtime.h>

namespace btam {

// relaxation (L-BFGS on occupancy-scaled z = (q, log sigma) of the real sites)
struct RelaxBounds {
  double ls_lo, ls_hi;  // log sigma bounds
  double x_min;         // sites with smaller occupancy are held fixed
};
cudaError_t relax_gather(int n, const double4 *pos, const double2 *xb, const double *V0,
                         const double *Rq, const double *Rs, const RelaxBounds &bd, double *z,
                         double *g, double *fterm, double *rterm, double *f_out,
                         double *r2_out, const double *ones, cudaStream_t st);
cudaError_t relax_apply(int n, const double2 *xb, const double *z0, const double *p,
                        double alpha, const RelaxBounds &bd, double4 *pos, cudaStream_t st);
cudaError_t vec_dot(int n, const double *a, const double *b, double *out, cudaStream_t st);
// out = a x + b y (out may alias x or y)
cudaError_t vec_axpby(int n, double a, const double *x, double b, const double *y, double *out,
                      cudaStream_t st);
cudaError_t lbfgs_direction(int n4, const double *g, double *const *S, double *const *Y,
                            const double *rho, const int *order, int m_used, double *p,
                            double *work_q, double *alpha, double *tmp, cudaStream_t st);
cudaError_t lbfgs_push(int n4, const double *z_new, const double *z_old, const double *g_new,
                       const double *g_old, double *S, double *Y, double *sy, cudaStream_t st);

// master equation
constexpr double kDmdQuantum = 8.8817841970012523e-16;    // 2^-50
constexpr double kDmdInvQuantum = 1125899906842624.0;     // 2^50

struct DmdParams {
  double dt;      // time step
  double Df;      // diffusivity (Variables.hpp:71)
  double dr;      // diffusive distance (Variables.hpp:77)
  double min_dx;  // smallest occupancy moved across an edge (Variables.hpp:85)
  double max_x;   // largest occupancy a site may receive up to (Variables.hpp:92)
};

struct DmdArgs {
  int n;  // real sites
  double2 *xb;
  const int *code, *owner;
  const double *Rx, *gamma;
  const int *moffs, *midx;  // mechanical neighbours (real sites)
  const int *doffs, *didx;  // diffusive neighbours (real sites)
  long long *X, *X0;        // occupancy quanta, snapshot
  double *mu;
  int *active, *deg;
  // step-control counters: [0] the largest edge move over its room and [1]
  // the largest site change over max_dx of the last decision (non-negative
  // doubles as their bits), [2] edge moves clipped to a nonzero room
  unsigned long long *ctl = nullptr;
};

cudaError_t dmd_init(int n, const double2 *xb, const int *code, long long *X, cudaStream_t st);
// x of every real H site from its quanta
cudaError_t dmd_commit_all(int n, const int *code, const long long *X, double2 *xb,
                           cudaStream_t st);
cudaError_t dmd_step(const DmdArgs &a, const DmdParams &prm, cudaStream_t st);
// The step in its parts: chemical potentials, activity and degrees of the
// current state; then (optionally) the step-control decision for a step
// of prm.dt into ctl[0..1]; then the occupancy update of one step of
// prm.dt (snapshot, edge moves, commit).
cudaError_t dmd_prepare(const DmdArgs &a, cudaStream_t st);
cudaError_t dmd_control(const DmdArgs &a, const DmdParams &prm, double max_dx, cudaStream_t st);
cudaError_t dmd_apply(const DmdArgs &a, const DmdParams &prm, cudaStream_t st);
cudaError_t dmd_total(int n, const int *code, const long long *X, long long *out2,
                      cudaStream_t st);

}  // namespace btam
