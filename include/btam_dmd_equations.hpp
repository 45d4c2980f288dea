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
 *    system, in its order; indices from n on are the system's periodic
 *    images in its numbering (btam_ghosts_copy: the order in which the
 *    reference's DMSwarmCreateGhostAtoms appends them).  Rows beyond n of
 *    the caller's arrays are never read: an image takes its owner's state.
 *    The caller's `mf_rho`/`rho` arguments are not read (rho-bar is
 *    recomputed with the state); `specie` is not read (the system keeps its
 *    own species).
 *  - A value of site i depends on the state of i and of its neighbours
 *    N(i).  Every call compares that state (the system's own lists, images
 *    mapped to their owners, and the site u a derivative is taken for) with
 *    the evaluated state; on any difference the whole state is taken from
 *    the caller's arrays and the values are evaluated again.  Calls are
 *    serialised by a mutex, so OpenMP callers are safe.
 *  - The derivative slots return the reference's per-pair values, one term
 *    per (u, i) call: evaluate_DV0_i_Dq_j(u, i) is dV0_i/d(q_u, sigma_u),
 *    evaluate_DV0_i_Dxi_j(u, i) is dV0_i/dx_u, and likewise the
 *    non-mean-field gradient and the Hessian blocks (btam_mf_pair_terms,
 *    btam_pt_pair_terms, btam_mf_hessian_pairs).  i = u is the self term;
 *    for i != u the pair is found in u's list as the entry whose owner is
 *    i's owner and whose image shift is i's minus u's, so both the entry as
 *    u's list names it and the pair the reference evaluates for it (u's
 *    image in i's list, i real) give the same value.  A site i that does not
 *    neighbour u gives 0, as in the reference.  A caller assembles a
 *    residual by summing over i in {u} U N(u), images included, with its
 *    own weights (the device's btam_mf_eval weights by beta_i / beta_u).
 *  - The non-mean-field forms (evaluate_rho_i, evaluate_DV_i_Dq_j,
 *    evaluate_DV_i_DF, evaluate_D2V_i_Dq2_j) come from btam_pt_eval and
 *    btam_pt_pair_terms of the state.
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
 *    btam_mf_stress in the bound precision; evaluate_D2V0_i_Dmeanq2_j is
 *    FP64 whatever the bound precision.  Every slot of the table is served.
 *  - A caller compiled with MULTIPOLE_INTEGRAL, as the reference's rule
 *    switch selects it, gets the mean-field values and derivatives of the
 *    multipole rule (btam_mf_eval_multipole, btam_mf_pair_terms_multipole,
 *    btam_mf_hessian_pairs_multipole; FP64): with finite-difference
 *    Hessians when NUMERICAL_DERIVATIVES is defined (the reference's
 *    CMakeLists.txt defines it), analytic ones otherwise; the mean-field
 *    stretch derivative too (btam_mf_stress_multipole).  The
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
  int n = 0, n_ghost = 0;
  bool have_state = false;  // q, sigma, x below are the system's state
  bool valid = false;       // mean-field per-site values of that state
  bool pairs_valid = false; // mean-field per-pair terms
  bool pt_valid = false;    // non-mean-field per-site values
  bool ptp_valid = false;   // non-mean-field per-pair terms and Hessian blocks
  bool mfs_valid = false;   // mean-field stress
  bool mfh_valid = false;   // mean-field per-pair Hessian blocks
  int status = BTAM_OK;     // status of the last evaluation
  std::vector<double> q, sigma, x;  // the evaluated state (q row-major)
  std::vector<double> q_bind;       // positions at bind(): the stretch reference
  double F[3] = {1.0, 1.0, 1.0};    // stretch of the system's cell against them
  // the system's lists of the real sites, owners and image shifts of all
  // sites (real sites: themselves, shift 0)
  std::vector<int> offs, idx, owner, shift;
  std::vector<double> rho, V0, S0;         // per site
  std::vector<double> self5, slot5;        // dV0/d(q, sigma, x): i = u, list entries
  std::vector<double> pt_rho, pt_W, mf_W;  // per site
  std::vector<double> pt_self3, pt_slot3, pt_Hself, pt_Hslot, mf_Hself, mf_Hslot;
};

inline Cache &cache() {
  static Cache c;
  return c;
}

/* Binds a built system (neighbour lists built): evaluations use `precision`
 * (BTAM_FP64 or BTAM_FP32C).  beta and gamma are accepted for the
 * signature of earlier versions and not read: the per-pair values do not
 * depend on them. */
inline int bind(btam_system *s, int precision, const double *beta, const double *gamma) {
  (void)beta;
  (void)gamma;
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  int n_real = 0, n_ghost = 0;
  long long n_pairs = 0;
  int st = btam_system_info(s, &n_real, &n_ghost, &n_pairs);
  if (st != BTAM_OK) return st;
  c.sys = s;
  c.precision = precision;
  c.n = n_real;
  c.n_ghost = n_ghost;
  c.have_state = c.valid = c.pairs_valid = c.pt_valid = c.ptp_valid = c.mfs_valid =
      c.mfh_valid = false;
  c.F[0] = c.F[1] = c.F[2] = 1.0;
  const size_t n = (size_t)n_real, na = n + (size_t)n_ghost;
  // the lists (btam_neighbors_copy returns every list the system holds;
  // the real sites' come first)
  std::vector<int> offs_all(na + 1, 0), idx_all((size_t)(n_pairs > 0 ? n_pairs : 1));
  st = btam_neighbors_copy(s, offs_all.data(), idx_all.data(), (long long)idx_all.size());
  if (st != BTAM_OK) return st;
  c.offs.assign(offs_all.begin(), offs_all.begin() + n + 1);
  c.idx.assign(idx_all.begin(), idx_all.begin() + c.offs[n]);
  c.owner.resize(na);
  c.shift.assign(3 * na, 0);
  for (size_t j = 0; j < n; ++j) c.owner[j] = (int)j;
  if (n_ghost > 0) {
    std::vector<double> qg(3 * (size_t)n_ghost);
    st = btam_ghosts_copy(s, qg.data(), c.owner.data() + n, c.shift.data() + 3 * n);
    if (st != BTAM_OK) return st;
  }
  const size_t ns = c.idx.size();
  c.q.assign(3 * n, 0.0);
  c.sigma.assign(n, 0.0);
  c.x.assign(n, 0.0);
  c.rho.assign(n, 0.0);
  c.V0.assign(n, 0.0);
  c.S0.assign(n, 0.0);
  c.self5.assign(5 * n, 0.0);
  c.slot5.assign(5 * ns, 0.0);
  c.pt_rho.assign(n, 0.0);
  c.pt_W.assign(9 * n, 0.0);
  c.mf_W.assign(9 * n, 0.0);
  c.pt_self3.assign(3 * n, 0.0);
  c.pt_slot3.assign(3 * ns, 0.0);
  c.pt_Hself.assign(9 * n, 0.0);
  c.pt_Hslot.assign(9 * ns, 0.0);
  c.mf_Hself.assign(9 * n, 0.0);
  c.mf_Hslot.assign(9 * ns, 0.0);
  st = btam_system_get_state(s, c.q.data(), c.sigma.data(), c.x.data());
  c.have_state = st == BTAM_OK;
  c.q_bind = c.q;
  return st;
}

/* Status of the last evaluation the adapter ran (the table's functions have
 * no error channel, as in the reference). */
inline int last_status() { return cache().status; }

namespace detail {

// Real site of a caller index (a real site or an image), -1 if out of range.
inline int owner_of(const Cache &c, unsigned j) {
  return (size_t)j < c.owner.size() ? c.owner[j] : -1;
}

template <class M, class V>
inline bool same_site(const Cache &c, int j, const M &mean_q, const V *stdv_q, const V &xi) {
  if (j < 0 || j >= c.n) return true;
  for (int k = 0; k < 3; ++k)
    if (mean_q(j, k) != c.q[3 * (size_t)j + k]) return false;
  if (stdv_q && (*stdv_q)(j) != c.sigma[j]) return false;
  return xi(j) == c.x[j];
}

// Entry of u's list that is the pair (u, i): -1 for i = u (the self term),
// -2 when i does not neighbour u.  The entry's owner is i's owner and its
// image shift is i's minus u's, so an image u of a real site and the entry
// as u's owner lists it name the same pair.
inline long long entry_of(const Cache &c, unsigned u, unsigned i) {
  if (u == i) return -1;
  const int u0 = owner_of(c, u), i0 = owner_of(c, i);
  if (u0 < 0 || i0 < 0) return -2;
  const int *su = &c.shift[3 * (size_t)u], *si = &c.shift[3 * (size_t)i];
  for (int p = c.offs[u0]; p < c.offs[u0 + 1]; ++p) {
    const int j = c.idx[p];
    if (c.owner[j] != i0) continue;
    const int *sj = &c.shift[3 * (size_t)j];
    if (sj[0] == si[0] - su[0] && sj[1] == si[1] - su[1] && sj[2] == si[2] - su[2]) return p;
  }
  return -2;
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

enum {
  kMeanField = 1, kPairs = 2, kPoint = 4, kPointPairs = 8, kStress = 16, kMfHessian = 32
};

// Loads the caller's state when the state a value of site i (and its
// derivative for site u) depends on differs from the cache: u, i and i's
// neighbours in the system's lists (images as their owners).  Then
// evaluates what `what` asks for and is not yet evaluated.
template <class M, class V>
inline void refresh(Cache &c, unsigned u, unsigned i, const M &mean_q, const V *stdv_q,
                    const V &xi, int what) {
  const int i0 = owner_of(c, i);
  bool same = c.have_state && same_site(c, owner_of(c, u), mean_q, stdv_q, xi) &&
              same_site(c, i0, mean_q, stdv_q, xi);
  if (same && i0 >= 0)
    for (int p = c.offs[i0]; same && p < c.offs[i0 + 1]; ++p)
      same = same_site(c, c.owner[c.idx[p]], mean_q, stdv_q, xi);
  if (!same) {
    for (int j = 0; j < c.n; ++j) {
      for (int k = 0; k < 3; ++k) c.q[3 * (size_t)j + k] = mean_q(j, k);
      if (stdv_q) c.sigma[j] = (*stdv_q)(j);
      c.x[j] = xi(j);
    }
    c.valid = c.pairs_valid = c.pt_valid = c.ptp_valid = c.mfs_valid = c.mfh_valid = false;
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
  const long long ns = (long long)c.idx.size();
#if defined(MULTIPOLE_INTEGRAL)
  // the caller is built with the reference's other rule
  // (MgHx-mf-V-bulk.cpp:715-724), whose Hessians follow the same
  // `#ifdef NUMERICAL_DERIVATIVES` as Quadrature-Multipole.cpp:134
#ifdef NUMERICAL_DERIVATIVES
  const int rule = BTAM_MP_FD;
#else
  const int rule = BTAM_MP_ANALYTIC;
#endif
#endif
  if ((what & kMeanField) && !c.valid) {
#if defined(MULTIPOLE_INTEGRAL)
    c.status = btam_mf_eval_multipole(c.sys, rule, c.rho.data(), c.V0.data(), c.S0.data(),
                                      nullptr);
#else
    c.status = btam_mf_eval(c.sys, c.precision, c.rho.data(), c.V0.data(), c.S0.data(),
                            nullptr, nullptr, nullptr, nullptr);
#endif
    c.valid = c.status == BTAM_OK;
  }
  if ((what & kPairs) && !c.pairs_valid) {
#if defined(MULTIPOLE_INTEGRAL)
    c.status = btam_mf_pair_terms_multipole(c.sys, rule, c.self5.data(), c.slot5.data(), ns);
#else
    c.status = btam_mf_pair_terms(c.sys, c.precision, c.self5.data(), c.slot5.data(), ns);
#endif
    c.pairs_valid = c.status == BTAM_OK;
  }
  if ((what & kPoint) && !c.pt_valid) {
    c.status = btam_pt_eval(c.sys, c.pt_rho.data(), nullptr, nullptr, c.pt_W.data(), nullptr);
    c.pt_valid = c.status == BTAM_OK;
  }
  if ((what & kPointPairs) && !c.ptp_valid) {
    c.status = btam_pt_pair_terms(c.sys, c.pt_self3.data(), c.pt_slot3.data(),
                                  c.pt_Hself.data(), c.pt_Hslot.data(), ns);
    c.ptp_valid = c.status == BTAM_OK;
  }
  if ((what & kStress) && !c.mfs_valid) {
#if defined(MULTIPOLE_INTEGRAL)
    c.status = btam_mf_stress_multipole(c.sys, rule, c.mf_W.data(), nullptr);
#else
    c.status = btam_mf_stress(c.sys, c.precision, c.mf_W.data(), nullptr);
#endif
    c.mfs_valid = c.status == BTAM_OK;
  }
  if ((what & kMfHessian) && !c.mfh_valid) {
#if defined(MULTIPOLE_INTEGRAL)
    c.status = btam_mf_hessian_pairs_multipole(c.sys, rule, c.mf_Hself.data(),
                                               c.mf_Hslot.data(), ns);
#else
    c.status = btam_mf_hessian_pairs(c.sys, c.mf_Hself.data(), c.mf_Hslot.data(), ns);
#endif
    c.mfh_valid = c.status == BTAM_OK;
  }
}

// Component c of the per-pair value (u, i) of width w: the self term of u's
// owner, the list entry, 0 when i does not neighbour u, NaN when the values
// are not valid or an index is out of range.
inline double pair_value(const Cache &c, bool valid, const std::vector<double> &self,
                         const std::vector<double> &slot, int w, unsigned u, unsigned i,
                         int comp) {
  const int u0 = owner_of(c, u);
  if (!valid || u0 < 0 || owner_of(c, i) < 0) return NAN;
  const long long e = entry_of(c, u, i);
  if (e == -1) return self[(size_t)w * u0 + comp];
  if (e < 0) return 0.0;
  return slot[(size_t)w * e + comp];
}

// A stress W taken at q0 = q, at reference positions mean_q0, which must be
// the bound positions (the cell's stretch F maps them to q): W(a, b) / F_b.
template <class M>
inline Eigen::Matrix3d stress_at_q0(Cache &c, const std::vector<double> &Wq, bool valid,
                                    unsigned i, const M &mean_q0) {
  const int i0 = owner_of(c, i);
  bool ok = valid && i0 >= 0 && (int)i < c.n;
  auto bound = [&](int j) {
    if (j < 0 || j >= c.n) return true;
    for (int k = 0; k < 3; ++k)
      if (mean_q0(j, k) != c.q_bind[3 * (size_t)j + k]) return false;
    return true;
  };
  ok = ok && bound(i0);
  for (int p = ok ? c.offs[i0] : 0; ok && p < c.offs[i0 + 1]; ++p) ok = bound(c.owner[c.idx[p]]);
  if (valid && !ok) c.status = BTAM_ERR_ARG;
  Eigen::Matrix3d W;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) W(a, b) = ok ? Wq[9 * (size_t)i + 3 * a + b] / c.F[b] : NAN;
  return W;
}

inline double site_value(const Cache &c, bool valid, const std::vector<double> &v, unsigned i) {
  const int i0 = owner_of(c, i);
  return valid && i0 >= 0 ? v[i0] : NAN;
}

inline double rho_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &xi,
                    const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, i, i, mean_q, nullptr, xi, kPoint);
  return site_value(c, c.pt_valid, c.pt_rho, i);
}

inline Eigen::Vector3d DV_Dq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                             const Eigen::VectorXd &xi, const Eigen::VectorXd &,
                             const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, u, i, mean_q, nullptr, xi, kPointPairs);
  Eigen::Vector3d g;
  for (int k = 0; k < 3; ++k) g(k) = pair_value(c, c.ptp_valid, c.pt_self3, c.pt_slot3, 3, u, i, k);
  return g;
}

inline Eigen::Matrix3d D2V_Dq2(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                               const Eigen::VectorXd &xi, const Eigen::VectorXd &,
                               const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, u, i, mean_q, nullptr, xi, kPointPairs);
  Eigen::Matrix3d H;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      H(a, b) = pair_value(c, c.ptp_valid, c.pt_Hself, c.pt_Hslot, 9, u, i, 3 * a + b);
  return H;
}

inline Eigen::Matrix3d D2V0_Dmeanq2(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                                    const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                                    const Eigen::VectorXd &, const AtomicSpecie *,
                                    const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, kMfHessian);
  Eigen::Matrix3d H;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      H(a, b) = pair_value(c, c.mfh_valid, c.mf_Hself, c.mf_Hslot, 9, u, i, 3 * a + b);
  return H;
}

inline Eigen::Matrix3d DV_DF(unsigned i, const Eigen::MatrixXd &mean_q,
                             const Eigen::MatrixXd &mean_q0, const Eigen::VectorXd &xi,
                             const Eigen::VectorXd &, const AtomicSpecie *,
                             const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh<Eigen::MatrixXd, Eigen::VectorXd>(c, i, i, mean_q, nullptr, xi, kPoint);
  return stress_at_q0(c, c.pt_W, c.pt_valid, i, mean_q0);
}

inline Eigen::Matrix3d DV0_DF(unsigned i, const Eigen::MatrixXd &mean_q,
                              const Eigen::MatrixXd &mean_q0, const Eigen::VectorXd &stdv_q,
                              const Eigen::VectorXd &xi, const Eigen::VectorXd &,
                              const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, kStress);
  return stress_at_q0(c, c.mf_W, c.mfs_valid, i, mean_q0);
}

inline double mf_rho_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                       const Eigen::VectorXd &xi, const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, kMeanField);
  return site_value(c, c.valid, c.rho, i);
}

inline double V0_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                   const Eigen::VectorXd &xi, const Eigen::VectorXd &, const AtomicSpecie *,
                   const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, kMeanField);
  return site_value(c, c.valid, c.V0, i);
}

inline double S0_i(unsigned i, const Eigen::MatrixXd &mean_q, const Eigen::VectorXd &stdv_q,
                   const Eigen::VectorXd &xi, const Eigen::VectorXd &, const Eigen::VectorXd &,
                   const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, i, i, mean_q, &stdv_q, xi, kMeanField);
  return site_value(c, c.valid, c.S0, i);
}

inline Eigen::Vector3d DV0_Dmeanq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                                  const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                                  const Eigen::VectorXd &, const AtomicSpecie *,
                                  const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, kPairs);
  Eigen::Vector3d g;
  for (int k = 0; k < 3; ++k) g(k) = pair_value(c, c.pairs_valid, c.self5, c.slot5, 5, u, i, k);
  return g;
}

inline double DV0_Dstdvq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                         const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                         const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, kPairs);
  return pair_value(c, c.pairs_valid, c.self5, c.slot5, 5, u, i, 3);
}

inline Eigen::Vector4d DV0_Dq(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                              const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                              const Eigen::VectorXd &, const AtomicSpecie *,
                              const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, kPairs);
  Eigen::Vector4d g;
  for (int k = 0; k < 4; ++k) g(k) = pair_value(c, c.pairs_valid, c.self5, c.slot5, 5, u, i, k);
  return g;
}

inline double DV0_Dxi(unsigned u, unsigned i, const Eigen::MatrixXd &mean_q,
                      const Eigen::VectorXd &stdv_q, const Eigen::VectorXd &xi,
                      const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  refresh(c, u, i, mean_q, &stdv_q, xi, kPairs);
  return pair_value(c, c.pairs_valid, c.self5, c.slot5, 5, u, i, 4);
}

}  // namespace detail

/* The per-term table (potential_function, Macros.hpp:252-278) of the four
 * ADP terms, served by btam_term_eval on the tables bound here.  The
 * functions keep the reference's signatures and write what the reference's
 * write (MgHx-ADP.cpp:509-2434): 1 value for F and dF_dn, 3 for the
 * gradients, a zeroed 3x3 block for the Hessians.  Each call is one device
 * evaluation of one geometry; a caller with many geometries calls
 * btam_term_eval once for all of them instead. */
inline const btam_tables *&term_tables() {
  static const btam_tables *t = nullptr;
  return t;
}
inline void bind_tables(const btam_tables *t) { term_tables() = t; }

namespace detail {
template <int Term, int Fn>
void term_slot(int direction, double *out, const double *xi, const double *q,
               const AtomicSpecie *spc) {
  const int ns = Term < 2 ? 2 : 3;
  const int width = (Fn == 0 || Fn == 5) ? 1 : (Fn == 2 || Fn == 4) ? 9 : 3;
  double qq[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, xx[3] = {0, 0, 0}, r[9];
  int sp[3] = {0, 0, 0};
  for (int k = 0; k < 3 * ns; ++k) qq[k] = q[k];
  for (int k = 0; k < ns; ++k) {
    xx[k] = xi[k];
    sp[k] = (int)spc[k];
  }
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  c.status = btam_term_eval(term_tables(), Term, Fn, direction, 1, qq, xx, sp, r);
  for (int k = 0; k < width; ++k) out[k] = c.status == BTAM_OK ? r[k] : std::nan("");
}
template <int Term>
void term_value(double *out, const double *xi, const double *q, const AtomicSpecie *spc) {
  term_slot<Term, 0>(0, out, xi, q, spc);
}
template <int Term>
potential_function term_table() {
  potential_function f;
  f.F = term_value<Term>;
  f.dF_dq = term_slot<Term, 1>;
  f.d2F_dq2 = term_slot<Term, 2>;
  f.dF_dq_FD = term_slot<Term, 3>;
  f.d2F_dq2_FD = term_slot<Term, 4>;
  f.dF_dn = term_slot<Term, 5>;
  return f;
}
}  // namespace detail
}  // namespace btam_compat

/* Drop-ins for rho_ij_adp_MgHx_constructor (MgHx-ADP.cpp:509-522),
 * V_pair_ij_adp_MgHx_constructor (848-865), V_dipole_ij1j2_adp_MgHx_
 * constructor (1213-1230) and V_quadrupole_ij1j2_adp_MgHx_constructor
 * (1762-1777), served by the tables bound with btam_compat::bind_tables. */
inline potential_function btam_rho_ij_adp_MgHx_constructor() {
  return btam_compat::detail::term_table<0>();
}
inline potential_function btam_V_pair_ij_adp_MgHx_constructor() {
  return btam_compat::detail::term_table<1>();
}
inline potential_function btam_V_dipole_ij1j2_adp_MgHx_constructor() {
  return btam_compat::detail::term_table<2>();
}
inline potential_function btam_V_quadrupole_ij1j2_adp_MgHx_constructor() {
  return btam_compat::detail::term_table<3>();
}

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
