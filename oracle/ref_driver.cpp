// Test infrastructure only (never linked into the product library).
//
// C-ABI driver around the reference's OWN arithmetic, compiled unmodified
// from the reference tree against oracle/ref_shim (see oracle/Makefile):
//   src/ADP/MgHx-ADP.cpp            table loader + ADP per-term functions
//   src/ADP/MgHx-mf-V-bulk.cpp      mean-field per-site drivers
//   src/ADP/density.cpp             non-mean-field density
//   src/Numerical/cubic-spline.cpp  spline evaluation
//   src/Numerical/Quadrature-*.cpp  Gaussian measure + degree-3 rule
// The driver only marshals plain arrays into the Eigen-typed signatures and
// loops over sites in parallel (the reference uses OpenMP over sites,
// main-BT-AM.cpp:197).  It is
// used to pin the restated oracle (oracle/btam_oracle.cpp), to generate the
// golden fixtures in tests/golden/, and as the timed "reference" CPU arm.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "ADP/MgHx-ADP.hpp"
#include "ADP/MgHx-mf-V-bulk.hpp"
#include "ADP/density.hpp"
#include "Macros.hpp"
#include "Numerical/Quadrature-Hermitian-3th.hpp"
#include "Numerical/Quadrature-Hermitian-5th.hpp"
#include "Numerical/Quadrature-Measure.hpp"
#include "Numerical/cubic-spline.hpp"

// Process globals the reference defines in src/Variables.hpp:25-26, 95-97, 107.
PetscMPIInt rank_MPI = 0;
PetscMPIInt size_MPI = 1;
adpPotential adp_MgMg;
adpPotential adp_HH;
adpPotential adp_MgH;
double element_mass[112];

namespace {

// Parallel loop over sites with std::thread (the reference uses OpenMP over
// sites, main-BT-AM.cpp:197; this image has no OpenMP runtime).  Thread count:
// BTAM_REF_THREADS, else all hardware threads.  Static contiguous chunks.
int ref_threads() {
  const char *e = getenv("BTAM_REF_THREADS");
  int t = e ? atoi(e) : (int)std::thread::hardware_concurrency();
  return t > 0 ? t : 1;
}

void   parallel_for(int n, const std::function<void(int)> &fn) {
  int t = ref_threads();
  if (t > n) t = n;
  if (t <= 1) {
    for (int k = 0; k < n; ++k) fn(k);
    return;
  }
  std::vector<std::thread> th;
  for (int w = 0; w < t; ++w)
    th.emplace_back([&, w]() {
      int lo = (int)((long long)n * w / t), hi = (int)((long long)n * (w + 1) / t);
      for (int k = lo; k < hi; ++k) fn(k);
    });
  for (auto &x : th) x.join();
}

struct Sys {
  Eigen::MatrixXd q;
  Eigen::VectorXd sigma, x, rho, beta, gamma;
  AtomicSpecie *spc = nullptr;
  const int *offs = nullptr;
  const int *idx = nullptr;
  int n = 0;
};

void make_sys(Sys &s, int n, const double *q, const double *sigma,
              const double *x, const int *spc, const int *offs,
              const int *idx) {
  s.n = n;
  s.q = Eigen::MatrixXd(n, 3);
  s.sigma = Eigen::VectorXd(n);
  s.x = Eigen::VectorXd(n);
  s.rho = Eigen::VectorXd(n);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) s.q(i, k) = q[3 * i + k];
    s.sigma(i) = sigma ? sigma[i] : 0.0;
    s.x(i) = x[i];
    s.rho(i) = 0.0;
  }
  s.spc = (AtomicSpecie *)malloc(sizeof(AtomicSpecie) * (n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) s.spc[i] = (AtomicSpecie)spc[i];
  s.offs = offs;
  s.idx = idx;
}

AtomTopology topo(const Sys &s, int i) {
  AtomTopology t;
  t.numneigh = s.offs[i + 1] - s.offs[i];
  t.mech_neighs_ptr = s.idx + s.offs[i];
  return t;
}

CubicSpline *table(int id) {
  switch (id) {
  case 0: return &adp_MgMg.rho;
  case 1: return &adp_HH.rho;
  case 2: return &adp_MgMg.embed;
  case 3: return &adp_HH.embed;
  case 4: return &adp_MgMg.pair;
  case 5: return &adp_HH.pair;
  case 6: return &adp_MgH.pair;
  case 7: return &adp_MgMg.u;
  case 8: return &adp_HH.u;
  case 9: return &adp_MgH.u;
  case 10: return &adp_MgMg.w;
  case 11: return &adp_HH.w;
  case 12: return &adp_MgH.w;
  }
  return nullptr;
}

} // namespace

extern "C" {

// init_adp_MgHx x3 (MgHx-ADP.cpp:366-501), as main-BT-AM.cpp:108-110 does.
int ref_load_tables(const char *dir) {
  if (init_adp_MgHx(&adp_MgMg, MgMg, dir) != EXIT_SUCCESS) return 1;
  if (init_adp_MgHx(&adp_HH, HH, dir) != EXIT_SUCCESS) return 1;
  if (init_adp_MgHx(&adp_MgH, MgH, dir) != EXIT_SUCCESS) return 1;
  return 0;
}

double ref_element_mass(int z) { return element_mass[z]; }

// cubic_spline / d_cubic_spline / d2_cubic_spline (cubic-spline.cpp:84-128).
double ref_spline(int table_id, double r, int deriv) {
  CubicSpline *t = table(table_id);
  if (!t) return 0.0;
  if (deriv == 0) return cubic_spline(t, r);
  if (deriv == 1) return d_cubic_spline(t, r);
  return d2_cubic_spline(t, r);
}

int ref_table_size(int table_id, double *dx) {
  CubicSpline *t = table(table_id);
  if (!t) return 0;
  *dx = t->dx;
  return t->n;
}

// Copies one table's nine coefficient columns (a,b,c,d,db,dc,dd,ddc,ddd).
int ref_table_coeffs(int table_id, double *out9n) {
  CubicSpline *t = table(table_id);
  if (!t) return 0;
  const double *cols[9] = {t->a, t->b, t->c, t->d, t->db,
                           t->dc, t->dd, t->ddc, t->ddd};
  for (int c = 0; c < 9; ++c)
    for (int m = 0; m < t->n; ++m) out9n[c * t->n + m] = cols[c][m];
  return t->n;
}

// One pair/triplet quadrature of one ADP term with the reference's measure
// and rule: term 0 = rho_ij, 1 = V_pair_ij, 2 = V_dipole, 3 = V_quadrupole.
// mode 0 = value, 1 = d/dmean_q of slot `slot` (3 values), 2 = d/dsigma of
// slot, 3 = d/dx of slot.  nsites = 2 (pair) or 3 (triplet);
// coincident = 1 builds the j1 == j2 dof table (MgHx-mf-V-bulk.cpp:892-895).
int ref_quadrature(int term, int mode, int slot, int nsites, int coincident,
                   const double *q, const double *sigma, const double *x,
                   const int *spc, double *out) {
  potential_function f;
  switch (term) {
  case 0: f = rho_ij_adp_MgHx_constructor(); break;
  case 1: f = V_pair_ij_adp_MgHx_constructor(); break;
  case 2: f = V_dipole_ij1j2_adp_MgHx_constructor(); break;
  case 3: f = V_quadrupole_ij1j2_adp_MgHx_constructor(); break;
  default: return 1;
  }
  double qq[9], ss[3], xx[3];
  AtomicSpecie sp[3];
  for (int k = 0; k < 3 * nsites; ++k) qq[k] = q[k];
  for (int k = 0; k < nsites; ++k) {
    ss[k] = sigma[k];
    xx[k] = x[k];
    sp[k] = (AtomicSpecie)spc[k];
  }
  int dof2[4] = {1, 0, 0, 1};
  int dof3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (coincident) {
    dof3[5] = 1;
    dof3[7] = 1;
  }
  gaussian_measure_ctx m = fill_out_gaussian_measure(
      qq, ss, xx, sp, nsites == 2 ? dof2 : dof3, (unsigned)nsites);
  if (mode == 0) meanfield_integral_gh3th(out, f, &m);
  else if (mode == 1) meanfield_integral_gh_3th_dmq(slot, out, f, &m);
  else if (mode == 2) meanfield_integral_gh3th_dsq(slot, out, f, &m);
  else meanfield_integral_gh_3th_dxi(slot, out, f, &m);
  destroy_gaussian_measure(&m);
  return 0;
}

// One slot of the per-term plugin table (potential_function, Macros.hpp:
// 252-278) of one ADP term at one geometry, through the reference's own
// constructor: fn 0 = F, 1 = dF_dq, 2 = d2F_dq2, 3 = dF_dq_FD,
// 4 = d2F_dq2_FD, 5 = dF_dn; out holds up to 9 values.
int ref_term_eval(int term, int fn, int direction, int nsites, const double *q,
                  const double *x, const int *spc, double *out) {
  potential_function f;
  switch (term) {
  case 0: f = rho_ij_adp_MgHx_constructor(); break;
  case 1: f = V_pair_ij_adp_MgHx_constructor(); break;
  case 2: f = V_dipole_ij1j2_adp_MgHx_constructor(); break;
  case 3: f = V_quadrupole_ij1j2_adp_MgHx_constructor(); break;
  default: return 1;
  }
  AtomicSpecie sp[3];
  for (int k = 0; k < nsites; ++k) sp[k] = (AtomicSpecie)spc[k];
  for (int k = 0; k < 9; ++k) out[k] = 0.0;
  switch (fn) {
  case 0: f.F(out, x, q, sp); break;
  case 1: f.dF_dq(direction, out, x, q, sp); break;
  case 2: f.d2F_dq2(direction, out, x, q, sp); break;
  case 3: f.dF_dq_FD(direction, out, x, q, sp); break;
  case 4: f.d2F_dq2_FD(direction, out, x, q, sp); break;
  case 5: f.dF_dn(direction, out, x, q, sp); break;
  default: return 1;
  }
  return 0;
}

// The reference's 5th-degree rule over the pair measure (Quadrature-Hermitian-
// 5th.cpp:31-432) of a pair term (0 rho_ij, 1 V_pair_ij) at one geometry:
// mode 0 moment_1th_Vij_gaussian_measure_5th (1 value),
// 1 moment_1th_grad_f_gaussian_measure_5th_6d (dF_dq of direction, 3),
// 2 moment_1th_hess_f_gaussian_measure_5th_6d (d2F_dq2 of direction, 9).
int ref_quad5(int term, int mode, int direction, const double *q, const double *sigma,
              const double *x, const int *spc, double *out) {
  potential_function f;
  switch (term) {
  case 0: f = rho_ij_adp_MgHx_constructor(); break;
  case 1: f = V_pair_ij_adp_MgHx_constructor(); break;
  default: return 1;
  }
  double qq[6], ss[2], xx[2];
  AtomicSpecie sp[2];
  for (int k = 0; k < 6; ++k) qq[k] = q[k];
  for (int k = 0; k < 2; ++k) {
    ss[k] = sigma[k];
    xx[k] = x[k];
    sp[k] = (AtomicSpecie)spc[k];
  }
  int dof[4] = {1, 0, 0, 1};
  gaussian_measure_ctx ctx = fill_out_gaussian_measure(qq, ss, xx, sp, dof, 2);
  for (int k = 0; k < 9; ++k) out[k] = 0.0;
  if (mode == 0) moment_1th_Vij_gaussian_measure_5th(out, f, &ctx);
  else if (mode == 1) moment_1th_grad_f_gaussian_measure_5th_6d(direction, out, f, &ctx);
  else moment_1th_hess_f_gaussian_measure_5th_6d(direction, out, f, &ctx);
  destroy_gaussian_measure(&ctx);
  return 0;
}

// evaluate_mf_rho_i_adp_MgHx (MgHx-mf-V-bulk.cpp:708-787) for each listed site.
void ref_mf_rho(int n, const double *q, const double *sigma, const double *x,
                const int *spc, const int *offs, const int *idx,
                const int *sites, int nsites, double *out) {
  Sys s;
  make_sys(s, n, q, sigma, x, spc, offs, idx);
  parallel_for(nsites, [&](int k) {
    int i = sites[k];
    out[k] = evaluate_mf_rho_i_adp_MgHx(i, s.q, s.sigma, s.x, s.spc, topo(s, i));
  });
  free(s.spc);
}

// evaluate_V0_i_adp_MgHx (791-953); rho holds mean-field rho of every site.
void ref_V0(int n, const double *q, const double *sigma, const double *x,
            const int *spc, const double *rho, const int *offs, const int *idx,
            const int *sites, int nsites, double *out) {
  Sys s;
  make_sys(s, n, q, sigma, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  parallel_for(nsites, [&](int k) {
    int i = sites[k];
    out[k] = evaluate_V0_i_adp_MgHx(i, s.q, s.sigma, s.x, s.rho, s.spc, topo(s, i));
  });
  free(s.spc);
}

// evaluate_S0_i_adp_MgHx (957-1142).
void ref_S0(int n, const double *q, const double *sigma, const double *x,
            const int *spc, const double *rho, const double *beta,
            const double *gamma, const int *offs, const int *idx,
            const int *sites, int nsites, double *out) {
  Sys s;
  make_sys(s, n, q, sigma, x, spc, offs, idx);
  s.beta = Eigen::VectorXd(n);
  s.gamma = Eigen::VectorXd(n);
  for (int i = 0; i < n; ++i) {
    s.rho(i) = rho[i];
    s.beta(i) = beta[i];
    s.gamma(i) = gamma[i];
  }
  parallel_for(nsites, [&](int k) {
    int i = sites[k];
    out[k] = evaluate_S0_i_adp_MgHx(i, s.q, s.sigma, s.x, s.rho, s.beta,
                                    s.gamma, s.spc, topo(s, i));
  });
  free(s.spc);
}

// evaluate_DV0_i_Dq_u_MgHx (1823-2098) -> 4 values per (u, i) pair and
// evaluate_DV0_i_Dxi_u_adp_MgHx (2102-2325) -> 1 value per pair.
void ref_DV0_pairs(int n, const double *q, const double *sigma,
                   const double *x, const int *spc, const double *rho,
                   const int *offs, const int *idx, const int *u_list,
                   const int *i_list, int npairs, double *out4,
                   double *out_x) {
  Sys s;
  make_sys(s, n, q, sigma, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  parallel_for(npairs, [&](int k) {
    int u = u_list[k], i = i_list[k];
    if (out4) {
      Eigen::Vector4d g = evaluate_DV0_i_Dq_u_MgHx(u, i, s.q, s.sigma, s.x,
                                                   s.rho, s.spc, topo(s, i));
      for (int c = 0; c < 4; ++c) out4[4 * k + c] = g(c);
    }
    if (out_x)
      out_x[k] = evaluate_DV0_i_Dxi_u_adp_MgHx(u, i, s.q, s.sigma, s.x, s.rho,
                                               s.spc, topo(s, i));
  });
  free(s.spc);
}

// evaluate_rho_i_adp_MgHx_kokkos (density.cpp:44-104): the non-mean-field
// density the shipped main-BT-AM.cpp evaluates.
void ref_rho_nmf(int n, const double *q, const double *x, const int *spc,
                 const int *offs, const int *idx, const int *sites, int nsites,
                 double *out) {
  Sys s;
  make_sys(s, n, q, nullptr, x, spc, offs, idx);
  parallel_for(nsites, [&](int k) {
    int i = sites[k];
    out[k] = evaluate_rho_i_adp_MgHx_kokkos(i, s.q, s.x, s.spc, topo(s, i));
  });
  free(s.spc);
}

// evaluate_DV_i_Dq_u_adp_MgHx (MgHx-mf-V-bulk.cpp:147-330): the
// non-mean-field gradient dV_i/dq_u, 3 values per (u, i) pair; rho is the
// non-mean-field density of every site.
void ref_pt_DV_pairs(int n, const double *q, const double *x, const int *spc,
                     const double *rho, const int *offs, const int *idx, const int *u_list,
                     const int *i_list, int npairs, double *out3) {
  Sys s;
  make_sys(s, n, q, nullptr, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  parallel_for(npairs, [&](int k) {
    int u = u_list[k], i = i_list[k];
    Eigen::Vector3d g = evaluate_DV_i_Dq_u_adp_MgHx(u, i, s.q, s.x, s.rho, s.spc, topo(s, i));
    for (int c = 0; c < 3; ++c) out3[3 * k + c] = g(c);
  });
  free(s.spc);
}

// evaluate_DV_i_dF_MgHx (MgHx-mf-V-bulk.cpp:530-704): 9 values per site,
// row-major, with reference positions q0 of every site.
void ref_pt_DV_dF(int n, const double *q, const double *q0, const double *x, const int *spc,
                  const double *rho, const int *offs, const int *idx, const int *sites,
                  int nsites, double *out9) {
  Sys s;
  make_sys(s, n, q, nullptr, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  Eigen::MatrixXd Q0(n, 3);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) Q0(i, k) = q0[3 * i + k];
  parallel_for(nsites, [&](int k) {
    int i = sites[k];
    Eigen::Matrix3d g = evaluate_DV_i_dF_MgHx(i, s.q, Q0, s.x, s.rho, s.spc, topo(s, i));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out9[9 * k + 3 * a + b] = g(a, b);
  });
  free(s.spc);
}

// evaluate_DV0_i_dF_bulk_MgHx (MgHx-mf-V-bulk.cpp:2329-2552): 9 values per
// site, row-major, with reference positions q0 of every site; rho is the
// mean-field density of every site.
void ref_mf_DV0_dF(int n, const double *q, const double *q0, const double *sigma,
                   const double *x, const int *spc, const double *rho, const int *offs,
                   const int *idx, const int *sites, int nsites, double *out9) {
  Sys s;
  make_sys(s, n, q, sigma, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  Eigen::MatrixXd Q0(n, 3);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) Q0(i, k) = q0[3 * i + k];
  parallel_for(nsites, [&](int k) {
    int i = sites[k];
    Eigen::Matrix3d g =
        evaluate_DV0_i_dF_bulk_MgHx(i, s.q, Q0, s.sigma, s.x, s.rho, s.spc, topo(s, i));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out9[9 * k + 3 * a + b] = g(a, b);
  });
  free(s.spc);
}

// evaluate_D2V_i_Dq2_u_MgHx (MgHx-mf-V-bulk.cpp:333-528): 9 values per
// (u, i) pair, row-major; rho is the non-mean-field density of every site.
void ref_pt_D2V_pairs(int n, const double *q, const double *x, const int *spc,
                      const double *rho, const int *offs, const int *idx, const int *u_list,
                      const int *i_list, int npairs, double *out9) {
  Sys s;
  make_sys(s, n, q, nullptr, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  parallel_for(npairs, [&](int k) {
    int u = u_list[k], i = i_list[k];
    Eigen::Matrix3d g = evaluate_D2V_i_Dq2_u_MgHx(u, i, s.q, s.x, s.rho, s.spc, topo(s, i));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out9[9 * k + 3 * a + b] = g(a, b);
  });
  free(s.spc);
}

// evaluate_D2V0_i_Dmeanq2_u_MgHx (MgHx-mf-V-bulk.cpp:1366-1600): 9 values per
// (u, i) pair, row-major; rho is the mean-field density of every site.
void ref_mf_D2V0_pairs(int n, const double *q, const double *sigma, const double *x,
                       const int *spc, const double *rho, const int *offs, const int *idx,
                       const int *u_list, const int *i_list, int npairs, double *out9) {
  Sys s;
  make_sys(s, n, q, sigma, x, spc, offs, idx);
  for (int i = 0; i < n; ++i) s.rho(i) = rho[i];
  parallel_for(npairs, [&](int k) {
    int u = u_list[k], i = i_list[k];
    Eigen::Matrix3d g =
        evaluate_D2V0_i_Dmeanq2_u_MgHx(u, i, s.q, s.sigma, s.x, s.rho, s.spc, topo(s, i));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out9[9 * k + 3 * a + b] = g(a, b);
  });
  free(s.spc);
}

} // extern "C"
