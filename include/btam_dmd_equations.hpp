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
 *  - The non-mean-field gradient, the Hessians and the stretch derivatives
 *    (evaluate_DV_i_Dq_j, evaluate_D2V_i_Dq2_j, evaluate_DV_i_DF,
 *    evaluate_D2V0_i_Dmeanq2_j, evaluate_DV0_i_DF) are not provided: their
 *    slots are null. */
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
  bool valid = false, nmf_valid = false;
  int status = BTAM_OK;  // status of the last evaluation
  std::vector<double> beta, gamma;
  std::vector<double> q, sigma, x;  // the evaluated state (q row-major)
  std::vector<double> rho, V0, S0, Rq, Rs, Rx, rho_nmf;
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
  c.valid = c.nmf_valid = false;
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
  c.rho_nmf.assign(n_real, 0.0);
  return btam_system_get_state(s, c.q.data(), c.sigma.data(), c.x.data());
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

// Re-evaluates when the sites a value depends on differ from the cache.
template <class M, class V>
inline void refresh(Cache &c, unsigned a, unsigned b, const M &mean_q, const V *stdv_q,
                    const V &xi, const AtomTopology &topo, bool nmf) {
  bool same = c.valid && same_site(c, (int)a, mean_q, stdv_q, xi) &&
              same_site(c, (int)b, mean_q, stdv_q, xi);
  for (int k = 0; same && k < topo.numneigh; ++k)
    same = same_site(c, (int)topo.mech_neighs_ptr[k], mean_q, stdv_q, xi);
  if (same && (!nmf || c.nmf_valid)) return;
  if (!same) {
    for (int j = 0; j < c.n; ++j) {
      for (int k = 0; k < 3; ++k) c.q[3 * (size_t)j + k] = mean_q(j, k);
      if (stdv_q) c.sigma[j] = (*stdv_q)(j);
      c.x[j] = xi(j);
    }
    c.status = btam_system_set_state(c.sys, c.q.data(), c.sigma.data(), c.x.data());
    c.valid = c.nmf_valid = false;
  }
  if (c.status == BTAM_OK && !c.valid) {
    c.status = btam_mf_eval(c.sys, c.precision, c.rho.data(), c.V0.data(), c.S0.data(),
                            c.Rq.data(), c.Rs.data(), c.Rx.data(), nullptr);
    c.valid = c.status == BTAM_OK;
  }
  if (nmf && c.status == BTAM_OK && !c.nmf_valid) {
    c.status = btam_rho_nmf(c.sys, c.rho_nmf.data());
    c.nmf_valid = c.status == BTAM_OK;
  }
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
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, i, i, mean_q, nullptr, xi, topo, true);
  return c.nmf_valid && (int)i < c.n ? c.rho_nmf[i] : NAN;
}

inline double mf_rho_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                       const Eigen::VectorXd &xi, const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, false);
  return c.valid && (int)i < c.n ? c.rho[i] : NAN;
}

inline double V0_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                   const Eigen::VectorXd &xi, const Eigen::VectorXd &, const AtomicSpecie *,
                   const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, false);
  return c.valid && (int)i < c.n ? c.V0[i] : NAN;
}

inline double S0_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                   const Eigen::VectorXd &xi, const Eigen::VectorXd &, const Eigen::VectorXd &,
                   const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, topo, false);
  return c.valid && (int)i < c.n ? c.S0[i] : NAN;
}

inline Eigen::Vector3d DV0_Dmeanq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                                  const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                                  const Eigen::VectorXd &, const AtomicSpecie *,
                                  const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, false);
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
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, false);
  if (!c.valid || (int)u >= c.n) return NAN;
  return u == i ? dV0_dsigma(c, (int)u) : 0.0;
}

inline Eigen::Vector4d DV0_Dq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                              const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                              const Eigen::VectorXd &, const AtomicSpecie *,
                              const AtomTopology topo) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, false);
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
  refresh(c, u, i, mean_q, &stdv_q, xi, topo, false);
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
  eq.evaluate_DV_i_Dq_j = nullptr;
  eq.evaluate_D2V_i_Dq2_j = nullptr;
  eq.evaluate_DV_i_DF = nullptr;
  eq.evaluate_mf_rho_i = d::mf_rho_i;
  eq.evaluate_V0_i = d::V0_i;
  eq.evaluate_S0_i = d::S0_i;
  eq.evaluate_DV0_i_Dmeanq_j = d::DV0_Dmeanq;
  eq.evaluate_D2V0_i_Dmeanq2_j = nullptr;
  eq.evaluate_DV0_i_Dstdvq_j = d::DV0_Dstdvq;
  eq.evaluate_DV0_i_Dq_j = d::DV0_Dq;
  eq.evaluate_DV0_i_Dxi_j = d::DV0_Dxi;
  eq.evaluate_DV0_i_DF = nullptr;
  return eq;
}

#endif
