// Device-resident relaxation of (q, sigma) and the hydrogen master-equation
// step: the two consumers of the residual evaluation.
//
// The reference has neither (its only solver, mechanical_relaxation_bulk in
// Mechanical-Relaxation-bulk.cpp:123-437, relaxes three stretches of the
// deformation gradient; the master equation exists only as parameters,
// src/Variables.hpp:68-90, and the diffusive graph, Neighbors.cpp:139-275).
// Both are defined here and restated by the CPU oracle.
//
// Relaxation: minimise  F(q, s) = sum_i beta_i V0_i - 3 sum_u log sigma_u,
// s = log sigma, over the active real sites; dF/dq_u = beta_u R_q(u) and
// dF/ds_u = beta_u sigma_u R_sigma(u), so F is stationary exactly where the
// residuals vanish.  Limited-memory BFGS (m pairs) with a backtracking
// Armijo line search; the vectors stay on the device, the host only reads
// two scalars per line-search trial.  Converged when
// sqrt(sum |R_q|^2 + R_sigma^2) <= tol.
#include <cuda_runtime.h>

#include <vector>

#include "solvers.cuh"

namespace btam {

namespace {

constexpr int kRB = 1024;  // threads of the single-block reductions

// Deterministic single-block reduction of sum a[i] * b[i] (fixed strides,
// fixed tree).
__global__ void __launch_bounds__(kRB) dot_kernel(int n, const double *a, const double *b,
                                                  double *out) {
  __shared__ double sh[kRB];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += kRB) v += a[i] * b[i];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = kRB / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// Per-site scale of the optimisation variables: a site's energy terms carry
// its occupancy, so its curvature does too; w = sqrt(max(x, 1e-3)) z puts
// weakly and fully occupied sites on a comparable footing.
__device__ __forceinline__ double occ_scale(double x) { return sqrt(fmax(x, 1e-3)); }

// w = scale (q, log sigma) of the real sites; gw = (beta R_q, beta sigma
// R_sigma) / scale on relaxed sites (x >= x_min), 0 elsewhere and on log
// sigma components pinned at a bound with the gradient pointing outwards;
// F = sum_active beta V0 - 3 sum_relaxed log sigma; the projected residual
// |R|^2 over the relaxed sites.
__global__ void gather_kernel(int n, const double4 *pos, const double2 *xb, const double *V0,
                              const double *Rq, const double *Rs, RelaxBounds bd, double *z,
                              double *g, double *fterm, double *rterm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = pos[i];
  double2 b = xb[i];
  bool act = b.x >= 5e-4;
  bool rel = act && b.x >= bd.x_min;
  double sc = occ_scale(b.x), ls = log(p.w), be = b.y;
  z[4 * i] = sc * p.x;
  z[4 * i + 1] = sc * p.y;
  z[4 * i + 2] = sc * p.z;
  z[4 * i + 3] = sc * ls;
  double gs = be * p.w * Rs[i];
  bool pin = (ls >= bd.ls_hi - 1e-12 && gs < 0.0) || (ls <= bd.ls_lo + 1e-12 && gs > 0.0);
  g[4 * i] = rel ? be * Rq[3 * i] / sc : 0.0;
  g[4 * i + 1] = rel ? be * Rq[3 * i + 1] / sc : 0.0;
  g[4 * i + 2] = rel ? be * Rq[3 * i + 2] / sc : 0.0;
  g[4 * i + 3] = (rel && !pin) ? gs / sc : 0.0;
  fterm[i] = act ? be * V0[i] - (rel ? 3.0 * ls : 0.0) : 0.0;
  rterm[i] = rel ? Rq[3 * i] * Rq[3 * i] + Rq[3 * i + 1] * Rq[3 * i + 1] +
                       Rq[3 * i + 2] * Rq[3 * i + 2] + (pin ? 0.0 : Rs[i] * Rs[i])
                 : 0.0;
}

// pos of real sites from w = w0 + alpha p (sigma = exp(s), s kept in bounds)
__global__ void apply_kernel(int n, const double2 *xb, const double *z0, const double *p,
                             double alpha, RelaxBounds bd, double4 *pos) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = xb[i].x;
  if (!(x >= 5e-4 && x >= bd.x_min)) return;  // held fixed: position left untouched
  double sc = occ_scale(x);
  double4 q = pos[i];
  q.x = (z0[4 * i] + alpha * p[4 * i]) / sc;
  q.y = (z0[4 * i + 1] + alpha * p[4 * i + 1]) / sc;
  q.z = (z0[4 * i + 2] + alpha * p[4 * i + 2]) / sc;
  double ls = (z0[4 * i + 3] + alpha * p[4 * i + 3]) / sc;
  q.w = exp(fmin(fmax(ls, bd.ls_lo), bd.ls_hi));
  pos[i] = q;
}

__global__ void axpy_kernel(int n, const double *alpha, double sgn, const double *x, double *y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += sgn * (*alpha) * x[i];
}
__global__ void scale_kernel(int n, const double *num, const double *den, double *y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double d = *den;
    y[i] *= (d > 0.0) ? (*num) / d : 1.0;
  }
}
__global__ void diff_kernel(int n, const double *a, const double *b, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] - b[i];
}
__global__ void neg_kernel(int n, const double *a, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = -a[i];
}
// alpha_k = rho_k * (s_k . q) ; scalar helpers on device
__global__ void mul_kernel(const double *a, const double *b, double *out) {
  if (threadIdx.x == 0) *out = (*a) * (*b);
}
// beta_k = rho_k * (y_k . r); coefficient alpha_k - beta_k
__global__ void sub_scal_kernel(const double *a, const double *b, double *out) {
  if (threadIdx.x == 0) *out = (*a) - (*b);
}

inline int nb(long long n) { return (int)((n + 255) / 256); }

}  // namespace

cudaError_t relax_gather(int n, const double4 *pos, const double2 *xb, const double *V0,
                         const double *Rq, const double *Rs, const RelaxBounds &bd, double *z,
                         double *g, double *fterm, double *rterm, double *f_out,
                         double *r2_out, const double *ones, cudaStream_t st) {
  gather_kernel<<<nb(n), 256, 0, st>>>(n, pos, xb, V0, Rq, Rs, bd, z, g, fterm, rterm);
  dot_kernel<<<1, kRB, 0, st>>>(n, fterm, ones, f_out);
  dot_kernel<<<1, kRB, 0, st>>>(n, rterm, ones, r2_out);
  return cudaGetLastError();
}

cudaError_t relax_apply(int n, const double2 *xb, const double *z0, const double *p,
                        double alpha, const RelaxBounds &bd, double4 *pos, cudaStream_t st) {
  apply_kernel<<<nb(n), 256, 0, st>>>(n, xb, z0, p, alpha, bd, pos);
  return cudaGetLastError();
}

namespace {
__global__ void axpby_kernel(int n, double a, const double *x, double b, const double *y,
                             double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a * x[i] + b * y[i];
}
}  // namespace

cudaError_t vec_axpby(int n, double a, const double *x, double b, const double *y, double *out,
                      cudaStream_t st) {
  if (n > 0) axpby_kernel<<<nb(n), 256, 0, st>>>(n, a, x, b, y, out);
  return cudaGetLastError();
}

cudaError_t vec_dot(int n, const double *a, const double *b, double *out, cudaStream_t st) {
  dot_kernel<<<1, kRB, 0, st>>>(n, a, b, out);
  return cudaGetLastError();
}

// Two-loop recursion: p = -H g from the stored pairs (s_k, y_k), newest last
// in `order`; all scalars stay on the device.
cudaError_t lbfgs_direction(int n4, const double *g, double *const *S, double *const *Y,
                            const double *rho, const int *order, int m_used, double *p,
                            double *work_q, double *alpha, double *tmp, cudaStream_t st) {
  cudaMemcpyAsync(work_q, g, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st);
  for (int t = m_used - 1; t >= 0; --t) {
    int k = order[t];
    dot_kernel<<<1, kRB, 0, st>>>(n4, S[k], work_q, tmp);
    mul_kernel<<<1, 32, 0, st>>>(rho + k, tmp, alpha + k);
    axpy_kernel<<<nb(n4), 256, 0, st>>>(n4, alpha + k, -1.0, Y[k], work_q);
  }
  if (m_used > 0) {
    int k = order[m_used - 1];
    // H0 = (s.y)/(y.y) I
    dot_kernel<<<1, kRB, 0, st>>>(n4, S[k], Y[k], tmp);
    dot_kernel<<<1, kRB, 0, st>>>(n4, Y[k], Y[k], tmp + 1);
    scale_kernel<<<nb(n4), 256, 0, st>>>(n4, tmp, tmp + 1, work_q);
  }
  for (int t = 0; t < m_used; ++t) {
    int k = order[t];
    dot_kernel<<<1, kRB, 0, st>>>(n4, Y[k], work_q, tmp + 2);
    mul_kernel<<<1, 32, 0, st>>>(rho + k, tmp + 2, tmp + 3);
    sub_scal_kernel<<<1, 32, 0, st>>>(alpha + k, tmp + 3, tmp + 4);
    axpy_kernel<<<nb(n4), 256, 0, st>>>(n4, tmp + 4, 1.0, S[k], work_q);
  }
  neg_kernel<<<nb(n4), 256, 0, st>>>(n4, work_q, p);
  return cudaGetLastError();
}

cudaError_t lbfgs_push(int n4, const double *z_new, const double *z_old, const double *g_new,
                       const double *g_old, double *S, double *Y, double *sy, cudaStream_t st) {
  diff_kernel<<<nb(n4), 256, 0, st>>>(n4, z_new, z_old, S);
  diff_kernel<<<nb(n4), 256, 0, st>>>(n4, g_new, g_old, Y);
  dot_kernel<<<1, kRB, 0, st>>>(n4, Y, S, sy);
  return cudaGetLastError();
}

}  // namespace btam

// ---------------------------------------------------------------------------
// Hydrogen master equation on the diffusive graph (H-H pairs within
// r_cutoff_Eb = 2.6 A, at most 50 per site: list_of_diffusive_neighs,
// Neighbors.cpp:139-275).  Occupancies are carried as int64 quanta of
// 2^-50, and every undirected edge moves +n quanta into one end and -n out
// of the other with integer atomics, so the total hydrogen is conserved
// exactly and the result does not depend on the order of the updates.
namespace btam {

namespace {

__global__ void dmd_init_kernel(int n, const double2 *xb, const int *code, long long *X) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  X[i] = code[i] == 1 ? llrint(xb[i].x * kDmdInvQuantum) : 0;
}

// chemical potential and diffusive activity (local H mass >= 0.01,
// Topology.cpp:202-364) of every real H site
__global__ void dmd_mu_kernel(int n, const double2 *xb, const int *code, const double *Rx,
                              const double *gamma, const int *moffs, const int *midx,
                              const long long *X, double *mu, int *active) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (code[i] != 1) {
    active[i] = 0;
    mu[i] = 0.0;
    return;
  }
  double x = (double)X[i] * kDmdQuantum, beta = xb[i].y;
  double mass = x;
  for (int p = moffs[i]; p < moffs[i + 1]; ++p) {
    int j = midx[p];
    if (code[j] == 1) mass += xb[j].x;
  }
  active[i] = mass >= 0.01 ? 1 : 0;
  if (x >= 5e-4) {
    mu[i] = Rx[i] + (x < 0.9999 ? gamma[i] / beta : 0.0);
  } else {
    double xt = x > 1e-12 ? x : 1e-12;
    mu[i] = -(3.0 / (2.0 * xt) + 1.0 / (1.0 - xt)) / beta;
  }
}

__global__ void dmd_degree_kernel(int n, const int *doffs, const int *didx, const int *owner,
                                  const int *active, int *deg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int d = 0;
  if (active[i])
    for (int p = doffs[i]; p < doffs[i + 1]; ++p) d += active[owner[didx[p]]];
  deg[i] = d;
}

// Occupancy moved from i to o across an active edge in one step: dt J with
// J = Df/dr^2 (beta_i+beta_j)/2 xm (1-xm) (mu_i - mu_o), xm = (x_i+x_o)/2
// (exactly antisymmetric in i, o).
__device__ __forceinline__ double dmd_move(const double2 *xb, const double *mu,
                                           const long long *X, int i, int o,
                                           const DmdParams &prm) {
  const double xi = (double)X[i] * kDmdQuantum, xo = (double)X[o] * kDmdQuantum;
  const double xm = 0.5 * (xi + xo), bm = 0.5 * (xb[i].y + xb[o].y);
  const double J = prm.Df / (prm.dr * prm.dr) * bm * xm * (1.0 - xm) * (mu[i] - mu[o]);
  return prm.dt * J;
}

// A move in quanta, rounded to nearest from a value first held within
// +-4e18 (far outside any room, which is at most max_x in quanta), so that a
// move whose quanta overflow 64 bits (an empty site's chemical potential
// against an occupied one) is cut to the room like any other large move.
__device__ __forceinline__ long long dmd_quanta(double dlt) {
  return llrint(fmin(fmax(dlt * kDmdInvQuantum, -4e18), 4e18));
}

// The room of edge (i, o) in quanta under the degree split: a move from i
// to o of at most hi, from o to i of at most -lo (lo <= 0).
__device__ __forceinline__ void dmd_room(const long long *X, const int *deg, int i, int o,
                                         long long xmax, long long &hi, long long &lo) {
  const long long di = deg[i] > 0 ? deg[i] : 1, dq = deg[o] > 0 ? deg[o] : 1;
  const long long out_i = X[i] / di, out_o = X[o] / dq;
  const long long in_i = xmax > X[i] ? (xmax - X[i]) / di : 0;
  const long long in_o = xmax > X[o] ? (xmax - X[o]) / dq : 0;
  hi = out_i < in_o ? out_i : in_o;
  lo = -(out_o < in_i ? out_o : in_i);
}

__global__ void dmd_flux_kernel(int n, const double2 *xb, const int *doffs, const int *didx,
                                const int *owner, const int *active, const int *deg,
                                const double *mu, const long long *X0, long long *X,
                                DmdParams prm, unsigned long long *ctl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !active[i]) return;
  const long long xmax = llrint(prm.max_x * kDmdInvQuantum);
  for (int p = doffs[i]; p < doffs[i + 1]; ++p) {
    int o = owner[didx[p]];
    if (o <= i || !active[o]) continue;  // each undirected edge once, from its lower end
    const double dlt = dmd_move(xb, mu, X0, i, o, prm);  // occupancy moved from i to o
    if (fabs(dlt) < prm.min_dx) continue;
    long long q = dmd_quanta(dlt);
    long long hi, lo;
    dmd_room(X0, deg, i, o, xmax, hi, lo);
    // a move cut to a nonzero room is counted; a zero room (empty giver,
    // full receiver) moves nothing and is not
    if (ctl && ((q > hi && hi > 0) || (q < lo && lo < 0))) atomicAdd(ctl + 2, 1ull);
    q = q > hi ? hi : (q < lo ? lo : q);
    if (q == 0) continue;
    atomicAdd((unsigned long long *)&X[i], (unsigned long long)(-q));
    atomicAdd((unsigned long long *)&X[o], (unsigned long long)q);
  }
}

// Step-control decision for a step of prm.dt at the current state: per
// site, its occupancy change over max_dx (moves below min_dx skipped, as in
// the update) and, over its edges to higher sites, each move over its
// nonzero room; the maxima go to ctl[1] and ctl[0] (a non-negative
// double's bits order as the double).
__global__ void dmd_control_kernel(int n, const double2 *xb, const int *doffs, const int *didx,
                                   const int *owner, const int *active, const int *deg,
                                   const double *mu, const long long *X, DmdParams prm,
                                   double max_dx, unsigned long long *ctl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ratio = 0.0, dx = 0.0;
  if (i < n && active[i]) {
    const long long xmax = llrint(prm.max_x * kDmdInvQuantum);
    for (int p = doffs[i]; p < doffs[i + 1]; ++p) {
      int o = owner[didx[p]];
      if (o == i || !active[o]) continue;
      const double dlt = dmd_move(xb, mu, X, i, o, prm);
      if (fabs(dlt) < prm.min_dx) continue;
      dx = __dsub_rn(dx, dlt);  // no contraction: the oracle rounds each term
      if (o < i) continue;  // the room of each edge once
      const long long q = dmd_quanta(dlt);
      long long hi, lo;
      dmd_room(X, deg, i, o, xmax, hi, lo);
      if (q > hi && hi > 0) ratio = fmax(ratio, (double)q / (double)hi);
      if (q < lo && lo < 0) ratio = fmax(ratio, (double)q / (double)lo);
    }
  }
  double r = fabs(dx) / max_dx;
  // warp maxima (every lane of the block takes part), then one atomic per warp
  for (int off = 16; off > 0; off >>= 1) {
    ratio = fmax(ratio, __shfl_xor_sync(0xffffffffu, ratio, off));
    r = fmax(r, __shfl_xor_sync(0xffffffffu, r, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(ctl, (unsigned long long)__double_as_longlong(ratio));
    atomicMax(ctl + 1, (unsigned long long)__double_as_longlong(r));
  }
}

__global__ void dmd_commit_kernel(int n, const int *code, const long long *X, double2 *xb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || code[i] != 1) return;
  xb[i].x = (double)X[i] * kDmdQuantum;
}

// exact total of the quanta (128-bit), single block, fixed order
__global__ void __launch_bounds__(1024) dmd_total_kernel(int n, const int *code,
                                                        const long long *X, long long *out) {
  __shared__ __int128 sh[1024];
  __int128 v = 0;
  for (int i = threadIdx.x; i < n; i += 1024)
    if (code[i] == 1) v += (__int128)X[i];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    unsigned __int128 u = (unsigned __int128)sh[0];
    out[0] = (long long)(u >> 64);
    out[1] = (long long)(unsigned long long)(u & 0xffffffffffffffffull);
  }
}

inline int nbk(long long n) { return (int)((n + 255) / 256); }

}  // namespace

cudaError_t dmd_init(int n, const double2 *xb, const int *code, long long *X, cudaStream_t st) {
  dmd_init_kernel<<<nbk(n), 256, 0, st>>>(n, xb, code, X);
  return cudaGetLastError();
}

cudaError_t dmd_commit_all(int n, const int *code, const long long *X, double2 *xb,
                           cudaStream_t st) {
  dmd_commit_kernel<<<nbk(n), 256, 0, st>>>(n, code, X, xb);
  return cudaGetLastError();
}

cudaError_t dmd_prepare(const DmdArgs &a, cudaStream_t st) {
  dmd_mu_kernel<<<nbk(a.n), 256, 0, st>>>(a.n, a.xb, a.code, a.Rx, a.gamma, a.moffs, a.midx,
                                          a.X, a.mu, a.active);
  dmd_degree_kernel<<<nbk(a.n), 256, 0, st>>>(a.n, a.doffs, a.didx, a.owner, a.active, a.deg);
  return cudaGetLastError();
}

cudaError_t dmd_control(const DmdArgs &a, const DmdParams &prm, double max_dx,
                        cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(a.ctl, 0, 2 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  dmd_control_kernel<<<nbk(a.n), 256, 0, st>>>(a.n, a.xb, a.doffs, a.didx, a.owner, a.active,
                                               a.deg, a.mu, a.X, prm, max_dx, a.ctl);
  return cudaGetLastError();
}

cudaError_t dmd_apply(const DmdArgs &a, const DmdParams &prm, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(a.X0, a.X, (size_t)a.n * sizeof(long long),
                                  cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  dmd_flux_kernel<<<nbk(a.n), 256, 0, st>>>(a.n, a.xb, a.doffs, a.didx, a.owner, a.active,
                                            a.deg, a.mu, a.X0, a.X, prm, a.ctl);
  dmd_commit_kernel<<<nbk(a.n), 256, 0, st>>>(a.n, a.code, a.X, a.xb);
  return cudaGetLastError();
}

cudaError_t dmd_step(const DmdArgs &a, const DmdParams &prm, cudaStream_t st) {
  cudaError_t e = dmd_prepare(a, st);
  return e == cudaSuccess ? dmd_apply(a, prm, st) : e;
}

cudaError_t dmd_total(int n, const int *code, const long long *X, long long *out2,
                      cudaStream_t st) {
  dmd_total_kernel<<<1, 1024, 0, st>>>(n, code, X, out2);
  return cudaGetLastError();
}

}  // namespace btam
