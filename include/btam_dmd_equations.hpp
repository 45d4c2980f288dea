/* Compatibility adapter: the reference's per-site plugin table served by
 * libbtam.
 *
 * The reference's mean-field equations are a table of function pointers,
 * `dmd_equations` (src/Macros.hpp:540-798), filled by DMD_MgHx_constructor()
 * (src/ADP/MgHx-mf-V-bulk.cpp:46-79) and called one site at a time from
 * OpenMP loops.  btam_DMD_MgHx_constructor() below returns the same table,
 * so a caller written against it links unchanged; the values come from one
 * whole-system evaluation on the device.
 *
 * Include this header after the reference's Macros.hpp (it uses the
 * reference's dmd_equations, AtomicSpecie, AtomTopology and Eigen types),
 * and link libbtam.so.  Then:
 *
 *   btam_system *S;  btam_system_create(...);  btam_neighbors_build(S, 0);
 *   btam_compat::bind(S, BTAM_FP64, beta, gamma);   // beta, gamma as created
 *   dmd_equations eq = btam_DMD_MgHx_constructor();
 *   ... the reference's per-site loops, unchanged ...
 *
 * Semantics:
 *  - Sites 0..n-1 of the caller's arrays are the real sites of the bound
 *    system, in its order; rows beyond n (the caller's ghost copies) are not
 *    read.  The caller's `mf_rho` is not read (rho-bar is recomputed with
 *    the state); `specie` is read only to tell H sites for the occupancy
 *    derivative (the system keeps its own species).
 *  - Every call compares the state of the sites it depends on (the site,
 *    the site whose derivative is asked for, and the neighbours in its
 *    AtomTopology) with the evaluated state; on any difference the whole
 *    state is taken from the caller's arrays and evaluated again.  Calls are
 *    serialised by a mutex, so OpenMP callers are safe.
 *  - The reference has no assembler of its per-pair derivatives (one term
 *    dV0_i/d(.)_u per call); the device computes the assembled residuals.
 *    So the derivative functions are lumped: for site_i == site_i_star they
 *    return the whole sum over i in {u} U N(u) of the terms the reference
 *    returns for (u, i), each weighted by beta_i / beta_u (plain sum when
 *    every site has the same beta), and zero for site_i != site_i_star.  A
 *    caller that sums over i, as every residual assembly does, gets the
 *    assembled value.  The occupancy derivative is defined for H sites
 *    (zero for Mg, as the device's R_x).
 *  - The non-mean-field forms (evaluate_rho_i, evaluate_DV_i_Dq_j,
 *    evaluate_DV_i_DF) come from one btam_pt_eval of the state; the
 *    gradient is lumped like the mean-field derivatives (the whole
 *    sum_{i in {u} U N(u)} dV_i/dq_u at site_i == site_i_star).  The
 *    caller's `rho` argument is not read.
 *  - Stretches: when the caller's mean_q is a diagonal stretch diag(F) of the
 *    positions bound with bind() (to 1e-13 relative, every row), the system's
 *    cell is stretched with it, so periodic images follow as the caller's
 *    stretched ghost rows do (Mechanical-Relaxation-bulk.cpp:505-520);
 *    any other mean_q is a new state in the current cell.
 *    evaluate_DV_i_DF and evaluate_DV0_i_DF are defined for mean_q0 equal
 *    to the bound positions (the reference's bulk residual passes its
 *    unstretched positions, Mechanical-Relaxation-bulk.cpp:577-579); other
 *    mean_q0 give NaN and last_status() BTAM_ERR_ARG.
 *  - evaluate_DV0_i_DF (the mean-field stretch derivative) comes from
 *    btam_mf_stress in the bound precision.
 *  - evaluate_D2V_i_Dq2_j (btam_pt_hessian) and evaluate_D2V0_i_Dmeanq2_j
 *    (btam_mf_hessian, FP64 whatever the bound precision) are lumped like
 *    the gradients: the whole sum over i in {u} U N(u) at site_i ==
 *    site_i_star.  Every slot of the table is served.
 *  - A caller compiled with MULTIPOLE_INTEGRAL, as the reference's rule
 *    switch selects it, gets the mean-field values and derivatives of the
 *    multipole rule (btam_mf_eval_multipole, btam_mf_residuals_multipole;
 *    FP64): with finite-difference Hessians when NUMERICAL_DERIVATIVES is
 *    defined (the reference's CMakeLists.txt defines it), analytic ones
 *    otherwise; the mean-field stretch derivative and Hessian blocks too
 *    (btam_mf_stress_multipole, btam_mf_hessian_multipole).  The
 *    non-mean-field forms have no rule. */
#ifndef BTAM_DMD_EQUATIONS_HPP
#define BTAM_DMD_EQUATIONS_HPP

#include <cmath>
#include <mutex>
#include <vector>

#include "btam.h"

namespace btam_compat {

struct Cache {
  std::mutex mu;
  btam_system *sys = nullptr;
  int precision = BTAM_FP64;
  int n = 0;
  bool have_state = false;  // q, sigma, x below are the system's state
  bool valid = false;       // mean-field results of that state
  bool pt_valid = false;    // non-mean-field results of that state
  bool mfs_valid = false;   // mean-field stress of that state
  bool pth_valid = false;   // non-mean-field Hessian blocks of that state
  bool mfh_valid = false;   // mean-field Hessian blocks of that state
  int status = BTAM_OK;     // status of the last evaluation
  std::vector<double> beta, gamma;
  std::vector<double> q, sigma, x;  // the evaluated state (q row-major)
  std::vector<double> q_bind;       // positions at bind(): the stretch reference
  double F[3] = {1.0, 1.0, 1.0};    // stretch of the system's cell against them
  std::vector<double> rho, V0, S0, Rq, Rs, Rx;
  std::vector<double> pt_rho, pt_Fq, pt_W, mf_W, pt_H, mf_H;
};

inline Cache &cache() {
  static Cache c;
  return c;
}

/* Binds a built system: evaluations use `precision` (BTAM_FP64 or
 * BTAM_FP32C); beta and gamma (n values each, NULL = the defaults of
 * btam_system_create) must be those the system was created with: the
 * adapter removes the entropy terms from the device's residuals with them. */
inline int bind(btam_system *s, int precision, const double *beta, const double *gamma) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  int n_real = 0, n_ghost = 0;
  long long n_pairs = 0;
  int st = btam_system_info(s, &n_real, &n_ghost, &n_pairs);
  if (st != BTAM_OK) return st;
  c.sys = s;
  c.precision = precision;
  c.n = n_real;
  c.have_state = c.valid = c.pt_valid = c.mfs_valid = c.pth_valid = c.mfh_valid = false;
  c.F[0] = c.F[1] = c.F[2] = 1.0;
  c.beta.assign(beta ? beta : nullptr, beta ? beta + n_real : nullptr);
  c.gamma.assign(gamma ? gamma : nullptr, gamma ? gamma + n_real : nullptr);
  if (!beta) c.beta.assign(n_real, 1.0 / (8.617332478e-5 * 300.0));  // k_B 300 K
  if (!gamma) c.gamma.assign(n_real, 0.0);
  c.q.assign(3 * (size_t)n_real, 0.0);
  c.sigma.assign(n_real, 0.0);
  c.x.assign(n_real, 0.0);
  c.rho.assign(n_real, 0.0);
  c.V0.assign(n_real, 0.0);
  c.S0.assign(n_real, 0.0);
  c.Rq.assign(3 * (size_t)n_real, 0.0);
  c.Rs.assign(n_real, 0.0);
  c.Rx.assign(n_real, 0.0);
  c.pt_rho.assign(n_real, 0.0);
  c.pt_Fq.assign(3 * (size_t)n_real, 0.0);
  c.pt_W.assign(9 * (size_t)n_real, 0.0);
  c.mf_W.assign(9 * (size_t)n_real, 0.0);
  c.pt_H.assign(9 * (size_t)n_real, 0.0);
  c.mf_H.assign(9 * (size_t)n_real, 0.0);
  st = btam_system_get_state(s, c.q.data(), c.sigma.data(), c.x.data());
  c.have_state = st == BTAM_OK;
  c.q_bind = c.q;
  return st;
}

/* Status of the last evaluation the adapter ran (the table's functions have
 * no error channel, as in the reference). */
inline int last_status() { return cache().status; }

namespace detail {

template <class M, class V>
inline bool same_site(const Cache &c, int j, const M &mean_q, const V *stdv_q, const V &xi) {
  if (j < 0 || j >= c.n) return true;
  for (int k = 0; k < 3; ++k)
    if (mean_q(j, k) != c.q[3 * (size_t)j + k]) return false;
  if (stdv_q && (*stdv_q)(j) != c.sigma[j]) return false;
  return xi(j) == c.x[j];
}

// Diagonal stretch F with c.q = diag(F) q_bind on every row (to 1e-13
// relative), fitted by least squares per component; false if none.
inline bool stretch_of(const Cache &c, double F[3]) {
  for (int k = 0; k < 3; ++k) {
    double num = 0.0, den = 0.0;
    for (int j = 0; j < c.n; ++j) {
      num += c.q[3 * (size_t)j + k] * c.q_bind[3 * (size_t)j + k];
      den += c.q_bind[3 * (size_t)j + k] * c.q_bind[3 * (size_t)j + k];
    }
    F[k] = den > 0.0 ? num / den : 1.0;
    if (!(F[k] > 0.0) || !std::isfinite(F[k])) return false;
    for (int j = 0; j < c.n; ++j) {
      const double v = c.q[3 * (size_t)j + k], b = F[k] * c.q_bind[3 * (size_t)j + k];
      if (std::fabs(v - b) > 1e-13 * (std::fabs(v) + 1.0)) return false;
    }
  }
  return true;
}

enum { kMeanField = 1, kPoint = 2, kStress = 4, kHessian = 8, kMfHessian = 16 };

// Loads the caller's state when the sites a value depends on differ from the
// cache, then evaluates what `what` asks for and is not yet evaluated.
template <class M, class V>
inline void refresh(Cache &c, unsigned a, unsigned b, const M &mean_q, const V *stdv_q,
                    const V &xi, const AtomTopology &topo, int what) {
  bool same = c.have_state && same_site(c, (int)a, mean_q, stdv_q, xi) &&
              same_site(c, (int)b, mean_q, stdv_q, xi);
  for (int k = 0; same && k < topo.numneigh; ++k)
    same = same_site(c, (int)topo.mech_neighs_ptr[k], mean_q, stdv_q, xi);
  if (!same) {
    for (int j = 0; j < c.n; ++j) {
      for (int k = 0; k < 3; ++k) c.q[3 * (size_t)j + k] = mean_q(j, k);
      if (stdv_q) c.sigma[j] = (*stdv_q)(j);
      c.x[j] = xi(j);
    }
    c.valid = c.pt_valid = c.mfs_valid = c.pth_valid = c.mfh_valid = false;
    // a stretch of the bound positions takes the cell with it; any other
    // state keeps the current cell
    double F[3];
    c.status = BTAM_OK;
    if (stretch_of(c, F) && (F[0] != c.F[0] || F[1] != c.F[1] || F[2] != c.F[2])) {
      const double rel[3] = {F[0] / c.F[0], F[1] / c.F[1], F[2] / c.F[2]};
      c.status = btam_stretch_apply(c.sys, rel);
      if (c.status == BTAM_OK)
        for (int k = 0; k < 3; ++k) c.F[k] = F[k];
    }
    if (c.status == BTAM_OK)
      c.status = btam_system_set_state(c.sys, c.q.data(), c.sigma.data(), c.x.data());
    c.have_state = c.status == BTAM_OK;
  }
  if (!c.have_state) return;
  if ((what & kMeanField) && !c.valid) {
#if defined(MULTIPOLE_INTEGRAL)
    // the caller is built with the reference's other rule
    // (MgHx-mf-V-bulk.cpp:715-724), whose Hessians follow the same
    // `#ifdef NUMERICAL_DERIVATIVES` as Quadrature-Multipole.cpp:134
#ifdef NUMERICAL_DERIVATIVES
    const int rule = BTAM_MP_FD;
#else
    const int rule = BTAM_MP_ANALYTIC;
#endif
    c.status = btam_mf_eval_multipole(c.sys, rule, c.rho.data(), c.V0.data(), c.S0.data(),
                                      nullptr);
    if (c.status == BTAM_OK)
      c.status = btam_mf_residuals_multipole(c.sys, rule, c.Rq.data(), c.Rs.data(), c.Rx.data());
#else
    c.status = btam_mf_eval(c.sys, c.precision, c.rho.data(), c.V0.data(), c.S0.data(),
                            c.Rq.data(), c.Rs.data(), c.Rx.data(), nullptr);
#endif
    c.valid = c.status == BTAM_OK;
  }
  if ((what & kPoint) && !c.pt_valid) {
    c.status = btam_pt_eval(c.sys, c.pt_rho.data(), nullptr, c.pt_Fq.data(), c.pt_W.data(),
                            nullptr);
    c.pt_valid = c.status == BTAM_OK;
  }
  if ((what & kStress) && !c.mfs_valid) {
#if defined(MULTIPOLE_INTEGRAL)
#ifdef NUMERICAL_DERIVATIVES
    c.status = btam_mf_stress_multipole(c.sys, BTAM_MP_FD, c.mf_W.data(), nullptr);
#else
    c.status = btam_mf_stress_multipole(c.sys, BTAM_MP_ANALYTIC, c.mf_W.data(), nullptr);
#endif
#else
    c.status = btam_mf_stress(c.sys, c.precision, c.mf_W.data(), nullptr);
#endif
    c.mfs_valid = c.status == BTAM_OK;
  }
  if ((what & kHessian) && !c.pth_valid) {
    c.status = btam_pt_hessian(c.sys, c.pt_H.data());
    c.pth_valid = c.status == BTAM_OK;
  }
  if ((what & kMfHessian) && !c.mfh_valid) {
#if defined(MULTIPOLE_INTEGRAL)
#ifdef NUMERICAL_DERIVATIVES
    c.status = btam_mf_hessian_multipole(c.sys, BTAM_MP_FD, c.mf_H.data());
#else
    c.status = btam_mf_hessian_multipole(c.sys, BTAM_MP_ANALYTIC, c.mf_H.data());
#endif
#else
    c.status = btam_mf_hessian(c.sys, c.mf_H.data());
#endif
    c.mfh_valid = c.status == BTAM_OK;
  }
}

// A stress W taken at q0 = q, at reference positions mean_q0, which must be
// the bound positions (the cell's stretch F maps them to q): W(a, b) / F_b.
template <class M>
inline Eigen::Matrix3d stress_at_q0(Cache &c, const std::vector<double> &Wq, bool valid,
                                    unsigned i, const M &mean_q0, const AtomTopology &topo) {
  bool ok = valid && (int)i < c.n;
  auto bound = [&](int j) {
    if (j < 0 || j >= c.n) return true;
    for (int k = 0; k < 3; ++k)
      if (mean_q0(j, k) != c.q_bind[3 * (size_t)j + k]) return false;
    return true;
  };
  ok = ok && bound((int)i);
  for (int k = 0; ok && k < topo.numneigh; ++k) ok = bound((int)topo.mech_neighs_ptr[k]);
  if (valid && !ok) c.status = BTAM_ERR_ARG;
  Eigen::Matrix3d W;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) W(a, b) = ok ? Wq[9 * (size_t)i + 3 * a + b] / c.F[b] : NAN;
  return W;
}

// Assembled sigma derivative of V0 (the residual without its entropy term
// -3 / (beta sigma)).
inline double dV0_dsigma(const Cache &c, int u) {
  return c.Rs[u] + 3.0 / (c.beta[u] * c.sigma[u]);
}

// Assembled occupancy derivative of V0 at an H site (R_x without its
// entropy and chemical terms); Mg sites (and empty sites) carry none.
inline double dV0_dx(const Cache &c, int u, bool hydrogen) {
  const double xu = c.x[u];
  if (!hydrogen || !(xu >= BTAM_MIN_OCCUPANCY)) return 0.0;
  const double dlogz = 3.0 / (2.0 * xu) + (xu < 1.0 ? 1.0 / (1.0 - xu) : 0.0);
  return c.Rx[u] + dlogz / c.beta[u] + (xu < 0.9999 ? c.gamma[u] / c.beta[u] : 0.0);
}

inline double rho_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &xi,
                    const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, i, i, mean_q, nullptr, xi, topo, kPoint);
  return c.pt_valid && (int)i < c.n ? c.pt_rho[i] : NAN;
}

inline Eigen::Vector3d DV_Dq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                             const Eigen::VectorXd &xi, const Eigen::VectorXd &,
                             const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, u, i, mean_q, nullptr, xi, topo, kPoint);
  Eigen::Vector3d g;
  for (int k = 0; k < 3; ++k)
    g(k) = !c.pt_valid || (int)u >= c.n ? NAN : (u == i ? c.pt_Fq[3 * (size_t)u + k] : 0.0);
  return g;
}

inline Eigen::Matrix3d D2V_Dq2(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                               const Eigen::VectorXd &xi, const Eigen::VectorXd &,
                               const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, u, i, mean_q, nullptr, xi, topo, kHessian);
  Eigen::Matrix3d H;
  const bool ok = c.pth_valid && (int)u < c.n;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      H(a, b) = !ok ? NAN : (u == i ? c.pt_H[9 * (size_t)u + 3 * a + b] : 0.0);
  return H;
}

inline Eigen::Matrix3d D2V0_Dmeanq2(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                                    const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                                    const Eigen::VectorXd &, const AtomicSpecie *,
                                    const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, kMfHessian);
  Eigen::Matrix3d H;
  const bool ok = c.mfh_valid && (int)u < c.n;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      H(a, b) = !ok ? NAN : (u == i ? c.mf_H[9 * (size_t)u + 3 * a + b] : 0.0);
  return H;
}

inline Eigen::Matrix3d DV_DF(unsigned i, const Eigen::MatrixXd &mean_q,
                             const Eigen::MatrixXd &mean_q0, const Eigen::VectorXd &xi,
                             const Eigen::VectorXd &, const AtomicSpecie *,
                             const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, i, i, mean_q, nullptr, xi, topo, kPoint);
  return stress_at_q0(c, c.pt_W, c.pt_valid, i, mean_q0, topo);
}

inline Eigen::Matrix3d DV0_DF(unsigned i, const Eigen::MatrixXd &mean_q,
                              const Eigen::MatrixXd &mean_q0, const Eigen::VectorXd &stdv_q,
                              const Eigen::VectorXd &xi, const Eigen::VectorXd &,
                              const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, kStress);
  return stress_at_q0(c, c.mf_W, c.mfs_valid, i, mean_q0, topo);
}

inline double mf_rho_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                       const Eigen::VectorXd &xi, const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, kMeanField);
  return c.valid && (int)i < c.n ? c.rho[i] : NAN;
}

inline double V0_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                   const Eigen::VectorXd &xi, const Eigen::VectorXd &, const AtomicSpecie *,
                   const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, kMeanField);
  return c.valid && (int)i < c.n ? c.V0[i] : NAN;
}

inline double S0_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                   const Eigen::VectorXd &xi, const Eigen::VectorXd &, const Eigen::VectorXd &,
                   const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, kMeanField);
  return c.valid && (int)i < c.n ? c.S0[i] : NAN;
}

inline Eigen::Vector3d DV0_Dmeanq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                                  const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                                  const Eigen::VectorXd &, const AtomicSpecie *,
                                  const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, kMeanField);
  Eigen::Vector3d g;
  for (int k = 0; k < 3; ++k)
    g(k) = !c.valid || (int)u >= c.n ? NAN : (u == i ? c.Rq[3 * (size_t)u + k] : 0.0);
  return g;
}

inline double DV0_Dstdvq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                         const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                         const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, kMeanField);
  if (!c.valid || (int)u >= c.n) return NAN;
  return u == i ? dV0_dsigma(c, (int)u) : 0.0;
}

inline Eigen::Vector4d DV0_Dq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                              const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                              const Eigen::VectorXd &, const AtomicSpecie *,
                              const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, kMeanField);
  Eigen::Vector4d g;
  const bool ok = c.valid && (int)u < c.n;
  for (int k = 0; k < 3; ++k) g(k) = !ok ? NAN : (u == i ? c.Rq[3 * (size_t)u + k] : 0.0);
  g(3) = !ok ? NAN : (u == i ? dV0_dsigma(c, (int)u) : 0.0);
  return g;
}

inline double DV0_Dxi(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                      const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                      const Eigen::VectorXd &, const AtomicSpecie *specie,
                      const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, kMeanField);
  if (!c.valid || (int)u >= c.n) return NAN;
  return u == i ? dV0_dx(c, (int)u, specie && (int)specie[u] == 1) : 0.0;  // 1: H
}

}  // namespace detail
}  // namespace btam_compat

/* Drop-in for DMD_MgHx_constructor() (MgHx-mf-V-bulk.cpp:46-79), served by
 * the system bound with btam_compat::bind. */
inline dmd_equations btam_DMD_MgHx_constructor() {
  namespace d = btam_compat::detail;
  dmd_equations eq;
  eq.evaluate_rho_i = d::rho_i;
  eq.evaluate_DV_i_Dq_j = d::DV_Dq;
  eq.evaluate_D2V_i_Dq2_j = d::D2V_Dq2;
  eq.evaluate_DV_i_DF = d::DV_DF;
  eq.evaluate_mf_rho_i = d::mf_rho_i;
  eq.evaluate_V0_i = d::V0_i;
  eq.evaluate_S0_i = d::S0_i;
  eq.evaluate_DV0_i_Dmeanq_j = d::DV0_Dmeanq;
  eq.evaluate_D2V0_i_Dmeanq2_j = d::D2V0_Dmeanq2;
  eq.evaluate_DV0_i_Dstdvq_j = d::DV0_Dstdvq;
  eq.evaluate_DV0_i_Dq_j = d::DV0_Dq;
  eq.evaluate_DV0_i_Dxi_j = d::DV0_Dxi;
  eq.evaluate_DV0_i_DF = d::DV0_DF;
  return eq;
}

#endif
