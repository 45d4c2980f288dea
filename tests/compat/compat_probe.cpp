// Test infrastructure only: a reference-style caller of the mean-field
// plugin table, built against the reference's type declarations (the
// oracle's shim of Macros.hpp) and include/btam_dmd_equations.hpp, linked
// with libbtam.so.  Reads a system from a binary file, evaluates it site by
// site through the table the way a residual assembly would (summing the
// per-pair derivatives over i in {u} U N(u), periodic images included, each
// call with the topology of site i), and writes the per-site values.
//
// Input (doubles unless noted): n (int), species (n ints), q (3n), sigma,
// x, beta, gamma (n each), origin (3), cell (9), periodic (3 ints).
// Output: per site rho, V0, S0, the sums over i of dV0_i/dq_u (3),
// dV0_i/dsigma_u and dV0_i/dx_u; then the status of the last evaluation.
//
// With the arguments `pt F0 F1 F2` after the output path, the probe runs
// the reference's bulk residual instead (evaluate_RHS,
// Mechanical-Relaxation-bulk.cpp:441-600) at mean_q = diag(F) q with
// mean_q0 = q: evaluate_rho_i over the sites, then per site the summed
// evaluate_DV_i_Dq_j, evaluate_DV_i_DF, the mean-field evaluate_DV0_i_DF and
// the summed evaluate_D2V_i_Dq2_j and evaluate_D2V0_i_Dmeanq2_j.  Output:
// per site rho, the gradient (3), dV/dF (9, row-major), dV0/dF (9), the
// Hessian block (9), the mean-field Hessian block (9); then Y (3) = sum_u
// diag(dV_u/dF) / V0 and the status.
//
// With the arguments `pairs <file>` after the output path, the probe calls
// the derivative slots one (u, i) pair at a time for the pairs the file
// lists (count (int), then u, i (ints) per pair; indices from n on are the
// system's periodic images) and writes per pair: evaluate_DV0_i_Dq_j (4),
// evaluate_DV0_i_Dxi_j, evaluate_DV0_i_Dmeanq_j (3),
// evaluate_DV0_i_Dstdvq_j, evaluate_DV_i_Dq_j (3), evaluate_D2V_i_Dq2_j (9),
// evaluate_D2V0_i_Dmeanq2_j (9); then the status.
//
// With the arguments `perturb u i j dq` after the output path, the probe
// reads evaluate_DV0_i_Dq_j and evaluate_DV0_i_Dxi_j of the pair (u, i),
// moves site j by dq along x in its own mean_q array, and reads the pair
// again: output 5 + 5 values, then the status.
//
// With `terms` as the only argument after the output path, the second
// argument is a file of term geometries instead of a system: count (int),
// then per row term, fn, direction (ints), q (9), x (3), species (3 ints).
// The probe calls the per-term table the reference's term constructors
// return (potential_function: F, dF_dq, d2F_dq2, dF_dq_FD, d2F_dq2_FD,
// dF_dn of rho_ij, V_pair_ij, V_dipole_ij1j2, V_quadrupole_ij1j2) through
// the btam_ drop-ins, one geometry per call, into a zeroed 9-value buffer
// per row, and writes the buffers; then the status.
#include "Macros.hpp"
#include "btam_dmd_equations.hpp"

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

static int run_terms(char **argv) {
  FILE *f = fopen(argv[2], "rb");
  if (!f) return 2;
  int m = 0;
  if (fread(&m, sizeof(int), 1, f) != 1) return 2;
  btam_tables *T = nullptr;
  int st = btam_tables_load(argv[1], &T);
  if (st != BTAM_OK) return 3;
  btam_compat::bind_tables(T);
  const potential_function tab[4] = {
      btam_rho_ij_adp_MgHx_constructor(), btam_V_pair_ij_adp_MgHx_constructor(),
      btam_V_dipole_ij1j2_adp_MgHx_constructor(),
      btam_V_quadrupole_ij1j2_adp_MgHx_constructor()};
  std::vector<double> out(9 * (size_t)m, 0.0);
  for (int r = 0; r < m && st == BTAM_OK; ++r) {
    int h[3], sp[3];
    double q[9], x[3];
    if (fread(h, sizeof(int), 3, f) != 3 || fread(q, sizeof(double), 9, f) != 9 ||
        fread(x, sizeof(double), 3, f) != 3 || fread(sp, sizeof(int), 3, f) != 3)
      return 2;
    AtomicSpecie spc[3] = {(AtomicSpecie)sp[0], (AtomicSpecie)sp[1], (AtomicSpecie)sp[2]};
    const potential_function &pf = tab[h[0]];
    double *o = out.data() + 9 * (size_t)r;
    switch (h[1]) {
      case 0: pf.F(o, x, q, spc); break;
      case 1: pf.dF_dq(h[2], o, x, q, spc); break;
      case 2: pf.d2F_dq2(h[2], o, x, q, spc); break;
      case 3: pf.dF_dq_FD(h[2], o, x, q, spc); break;
      case 4: pf.d2F_dq2_FD(h[2], o, x, q, spc); break;
      default: pf.dF_dn(h[2], o, x, q, spc); break;
    }
    st = btam_compat::last_status();
  }
  fclose(f);
  FILE *o = fopen(argv[3], "wb");
  if (!o) return 2;
  fwrite(out.data(), sizeof(double), out.size(), o);
  fwrite(&st, sizeof(int), 1, o);
  fclose(o);
  btam_tables_destroy(T);
  return 0;
}

int main(int argc, char **argv) {
  if (argc == 5 && std::string(argv[4]) == "terms") return run_terms(argv);
  const bool pt = argc == 8 && std::string(argv[4]) == "pt";
  const bool pairs = argc == 6 && std::string(argv[4]) == "pairs";
  const bool perturb = argc == 9 && std::string(argv[4]) == "perturb";
  if (argc != 4 && !pt && !pairs && !perturb) return 2;
  FILE *f = fopen(argv[2], "rb");
  if (!f) return 2;
  int n = 0;
  if (fread(&n, sizeof(int), 1, f) != 1) return 2;
  std::vector<int> spc(n), per(3);
  std::vector<double> q(3 * n), sigma(n), x(n), beta(n), gamma(n), origin(3), cell(9);
  bool ok = fread(spc.data(), sizeof(int), n, f) == (size_t)n &&
            fread(q.data(), sizeof(double), 3 * n, f) == (size_t)(3 * n) &&
            fread(sigma.data(), sizeof(double), n, f) == (size_t)n &&
            fread(x.data(), sizeof(double), n, f) == (size_t)n &&
            fread(beta.data(), sizeof(double), n, f) == (size_t)n &&
            fread(gamma.data(), sizeof(double), n, f) == (size_t)n &&
            fread(origin.data(), sizeof(double), 3, f) == 3 &&
            fread(cell.data(), sizeof(double), 9, f) == 9 &&
            fread(per.data(), sizeof(int), 3, f) == 3;
  fclose(f);
  if (!ok) return 2;
  btam_tables *T = nullptr;
  btam_system *S = nullptr;
  int st = btam_tables_load(argv[1], &T);
  if (st == BTAM_OK)
    st = btam_system_create(T, n, q.data(), sigma.data(), x.data(), spc.data(), beta.data(),
                            gamma.data(), origin.data(), cell.data(), per.data(), &S);
  if (st == BTAM_OK) st = btam_neighbors_build(S, 0);
  if (st == BTAM_OK) st = btam_compat::bind(S, BTAM_FP64, beta.data(), gamma.data());
  if (st != BTAM_OK) {
    fprintf(stderr, "set-up failed: %s\n", btam_status_string(st));
    return 1;
  }
  long long np = 0;
  int nr = 0, ng = 0;
  btam_system_info(S, &nr, &ng, &np);
  std::vector<int> offs(n + 1), idx(np > 0 ? np : 1);
  btam_neighbors_copy(S, offs.data(), idx.data(), (long long)idx.size());
  // owners of the images (numbered after the real sites)
  std::vector<int> owner(n + ng), shift(3 * (size_t)(ng > 0 ? ng : 1));
  std::vector<double> qg(3 * (size_t)(ng > 0 ? ng : 1));
  for (int i = 0; i < n; ++i) owner[i] = i;
  if (ng > 0) btam_ghosts_copy(S, qg.data(), owner.data() + n, shift.data());
  // each site's list as the reference's AtomTopology (an image's is its
  // owner's, translated)
  std::vector<std::vector<PetscInt>> nbs(n);
  for (int u = 0; u < n; ++u)
    for (int p = offs[u]; p < offs[u + 1]; ++p) nbs[u].push_back(idx[p]);
  auto topo_of = [&](unsigned i) {
    const int o = owner[i];
    return AtomTopology{(int)nbs[o].size(), nbs[o].data()};
  };
  // the caller's fields, as the reference holds them (the real sites' rows;
  // images are read through their owners)
  Eigen::MatrixXd mean_q(n, 3);
  Eigen::VectorXd stdv_q(n), xi(n), rho_v(n), beta_v(n), gamma_v(n);
  std::vector<AtomicSpecie> specie(n);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) mean_q(i, k) = q[3 * i + k];
    stdv_q(i) = sigma[i];
    xi(i) = x[i];
    beta_v(i) = beta[i];
    gamma_v(i) = gamma[i];
    specie[i] = (AtomicSpecie)spc[i];
  }
  dmd_equations eq = btam_DMD_MgHx_constructor();
  FILE *o = fopen(argv[3], "wb");
  if (!o) return 2;
  if (perturb) {
    const unsigned u = atoi(argv[5]), i = atoi(argv[6]);
    const int j = atoi(argv[7]);
    double v[10];
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) mean_q(j, 0) += atof(argv[8]);
      Eigen::Vector4d d = eq.evaluate_DV0_i_Dq_j(u, i, mean_q, stdv_q, xi, rho_v, specie.data(),
                                                 topo_of(i));
      for (int c = 0; c < 4; ++c) v[5 * pass + c] = d(c);
      v[5 * pass + 4] =
          eq.evaluate_DV0_i_Dxi_j(u, i, mean_q, stdv_q, xi, rho_v, specie.data(), topo_of(i));
    }
    fwrite(v, sizeof(double), 10, o);
    const int last = btam_compat::last_status();
    fwrite(&last, sizeof(int), 1, o);
    fclose(o);
    btam_system_destroy(S);
    btam_tables_destroy(T);
    return last == BTAM_OK ? 0 : 1;
  }
  if (pairs) {
    FILE *pf = fopen(argv[5], "rb");
    if (!pf) return 2;
    int m = 0;
    if (fread(&m, sizeof(int), 1, pf) != 1) return 2;
    std::vector<int> ui(2 * (size_t)m);
    if (fread(ui.data(), sizeof(int), ui.size(), pf) != ui.size()) return 2;
    fclose(pf);
    for (int k = 0; k < m; ++k) {
      const unsigned u = ui[2 * k], i = ui[2 * k + 1];
      const AtomTopology topo = topo_of(i);
      double v[30];
      Eigen::Vector4d d4 = eq.evaluate_DV0_i_Dq_j(u, i, mean_q, stdv_q, xi, rho_v,
                                                  specie.data(), topo);
      for (int c = 0; c < 4; ++c) v[c] = d4(c);
      v[4] = eq.evaluate_DV0_i_Dxi_j(u, i, mean_q, stdv_q, xi, rho_v, specie.data(), topo);
      Eigen::Vector3d d3 = eq.evaluate_DV0_i_Dmeanq_j(u, i, mean_q, stdv_q, xi, rho_v,
                                                      specie.data(), topo);
      for (int c = 0; c < 3; ++c) v[5 + c] = d3(c);
      v[8] = eq.evaluate_DV0_i_Dstdvq_j(u, i, mean_q, stdv_q, xi, rho_v, specie.data(), topo);
      Eigen::Vector3d g = eq.evaluate_DV_i_Dq_j(u, i, mean_q, xi, rho_v, specie.data(), topo);
      for (int c = 0; c < 3; ++c) v[9 + c] = g(c);
      Eigen::Matrix3d h = eq.evaluate_D2V_i_Dq2_j(u, i, mean_q, xi, rho_v, specie.data(), topo);
      Eigen::Matrix3d h0 = eq.evaluate_D2V0_i_Dmeanq2_j(u, i, mean_q, stdv_q, xi, rho_v,
                                                        specie.data(), topo);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          v[12 + 3 * a + b] = h(a, b);
          v[21 + 3 * a + b] = h0(a, b);
        }
      fwrite(v, sizeof(double), 30, o);
    }
    const int last = btam_compat::last_status();
    fwrite(&last, sizeof(int), 1, o);
    fclose(o);
    btam_system_destroy(S);
    btam_tables_destroy(T);
    return last == BTAM_OK ? 0 : 1;
  }
  if (pt) {
    const double F[3] = {atof(argv[5]), atof(argv[6]), atof(argv[7])};
    Eigen::MatrixXd q_ref = mean_q;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) mean_q(i, k) = F[k] * q_ref(i, k);
    const double vol = std::fabs(cell[0] * (cell[4] * cell[8] - cell[5] * cell[7]) -
                                 cell[1] * (cell[3] * cell[8] - cell[5] * cell[6]) +
                                 cell[2] * (cell[3] * cell[7] - cell[4] * cell[6]));
    for (int u = 0; u < n; ++u)
      rho_v(u) = eq.evaluate_rho_i(u, mean_q, xi, specie.data(), topo_of(u));
    double Y[3] = {0, 0, 0};
    for (int u = 0; u < n; ++u) {
      const AtomTopology topo_u = topo_of(u);
      double v[40];
      v[0] = rho_v(u);
      double g[3] = {0, 0, 0}, h[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      double h0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = -1; k < (int)nbs[u].size(); ++k) {
        const unsigned i = k < 0 ? u : nbs[u][k];
        const AtomTopology topo = topo_of(i);
        Eigen::Vector3d d = eq.evaluate_DV_i_Dq_j(u, i, mean_q, xi, rho_v, specie.data(), topo);
        for (int c = 0; c < 3; ++c) g[c] += d(c);
        Eigen::Matrix3d dd =
            eq.evaluate_D2V_i_Dq2_j(u, i, mean_q, xi, rho_v, specie.data(), topo);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) h[3 * a + b] += dd(a, b);
        Eigen::Matrix3d d0 = eq.evaluate_D2V0_i_Dmeanq2_j(u, i, mean_q, stdv_q, xi, rho_v,
                                                          specie.data(), topo);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) h0[3 * a + b] += d0(a, b);
      }
      for (int c = 0; c < 9; ++c) v[22 + c] = h[c];
      for (int c = 0; c < 9; ++c) v[31 + c] = h0[c];
      for (int c = 0; c < 3; ++c) v[1 + c] = g[c];
      Eigen::Matrix3d W = eq.evaluate_DV_i_DF(u, mean_q, q_ref, xi, rho_v, specie.data(), topo_u);
      for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) v[4 + 3 * a + b] = W(a, b);
        Y[a] += W(a, a) / vol;
      }
      Eigen::Matrix3d W0 =
          eq.evaluate_DV0_i_DF(u, mean_q, q_ref, stdv_q, xi, rho_v, specie.data(), topo_u);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) v[13 + 3 * a + b] = W0(a, b);
      fwrite(v, sizeof(double), 40, o);
    }
    fwrite(Y, sizeof(double), 3, o);
    const int last = btam_compat::last_status();
    fwrite(&last, sizeof(int), 1, o);
    fclose(o);
    btam_system_destroy(S);
    btam_tables_destroy(T);
    return last == BTAM_OK ? 0 : 1;
  }
  for (int u = 0; u < n; ++u) {
    const std::vector<PetscInt> &nb = nbs[u];
    const AtomTopology topo_u = topo_of(u);
    double v[8];
    v[0] = eq.evaluate_mf_rho_i(u, mean_q, stdv_q, xi, specie.data(), topo_u);
    rho_v(u) = v[0];
    v[1] = eq.evaluate_V0_i(u, mean_q, stdv_q, xi, rho_v, specie.data(), topo_u);
    v[2] = eq.evaluate_S0_i(u, mean_q, stdv_q, xi, rho_v, beta_v, gamma_v, specie.data(),
                            topo_u);
    // residual assembly over i in {u} U N(u), as a caller of the reference's
    // pair derivatives would write it
    double g[4] = {0, 0, 0, 0}, gx = 0;
    for (int k = -1; k < (int)nb.size(); ++k) {
      const unsigned i = k < 0 ? u : nb[k];
      const AtomTopology topo = topo_of(i);
      Eigen::Vector4d d = eq.evaluate_DV0_i_Dq_j(u, i, mean_q, stdv_q, xi, rho_v,
                                                 specie.data(), topo);
      for (int c = 0; c < 4; ++c) g[c] += d(c);
      gx += eq.evaluate_DV0_i_Dxi_j(u, i, mean_q, stdv_q, xi, rho_v, specie.data(), topo);
    }
    v[3] = g[0];
    v[4] = g[1];
    v[5] = g[2];
    v[6] = g[3];
    v[7] = gx;
    fwrite(v, sizeof(double), 8, o);
  }
  const int last = btam_compat::last_status();
  fwrite(&last, sizeof(int), 1, o);
  fclose(o);
  btam_system_destroy(S);
  btam_tables_destroy(T);
  return last == BTAM_OK ? 0 : 1;
}
