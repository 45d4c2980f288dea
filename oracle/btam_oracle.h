/* Test infrastructure only: the CPU oracle.  Nothing in the product library
 * links or calls this; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, to check results or to time the CPU path.
 *
 * A plain restatement of the reference's algorithm for the mean-field ADP
 * path (each function cites the reference file:line it follows), plus the
 * project-defined pieces the reference lacks (residual assembly, periodic
 * images done as the evident intent of Ghosts.cpp, master-equation step,
 * relaxation).  Parity of the restated arithmetic is pinned against the
 * reference's own files compiled unmodified (oracle/ref_driver.cpp) and
 * against the committed fixtures in tests/golden/.
 *
 * Species are atomic numbers as in the reference's AtomicSpecie enum
 * (H = 1, Mg = 12).  Positions are row-major N x 3 doubles. */
#ifndef BTAM_ORACLE_H
#define BTAM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Table ids: 0 rho_Mg, 1 rho_H, 2 F_Mg, 3 F_H, 4/5/6 phi MgMg/HH/MgH,
 * 7/8/9 u MgMg/HH/MgH, 10/11/12 w MgMg/HH/MgH. */
int orc_load_tables(const char *dir);
/* Integration rule of the mean-field forms: 0 the degree-3 Gauss-Hermite
 * rule (default, the reference's shipped build); 1 the multipole rule as
 * the reference's build flags compile it (-DMULTIPOLE_INTEGRAL with
 * -DNUMERICAL_DERIVATIVES=0: finite-difference Hessians); 2 the multipole
 * rule with analytic Hessians (NUMERICAL_DERIVATIVES undefined). */
void orc_set_rule(int rule);
double orc_spline(int table, double r, int deriv);
int orc_table_info(int table, double *dx);
double orc_mass(int species);

/* Periodic images of real sites within rc of the box (orthogonal box: the
 * slab rule of Ghosts.cpp:123-648 with the image shift the single-rank run
 * intends; triclinic box: the same rule in fractional coordinates).
 * cell[9] holds the three lattice vectors as rows (a1, a2, a3).
 * Returns 0, or an error code (see include/btam.h). */
int orc_ghosts(int n, const double *q, const double *origin, const double *cell,
               const int *periodic, double rc, int max_ghosts, double *q_ghost,
               int *owner, int *image, int *n_ghost);

/* Brute-force neighbour lists (Neighbors.cpp:39-134) for sites listed in
 * `query` against all n sites: ascending index, distance test
 * sqrt((dx^2+dy^2)+dz^2) <= rc in IEEE double.  offs has nquery+1 entries.
 * Returns 0, BTAM_ERR_NEIGHBOR_OVERFLOW or BTAM_ERR_NO_NEIGHBORS. */
int orc_neighbors(int n, const double *q, double rc, int maxn, const int *query,
                  int nquery, int *offs, int *idx, int idx_cap);

/* Quadrature of one ADP term (as ref_quadrature in oracle/ref_driver.cpp). */
int orc_quadrature(int term, int mode, int slot, int nsites, int coincident,
                   const double *q, const double *sigma, const double *x,
                   const int *spc, double *out);
/* One slot of the per-term table at one geometry (fn 0 F, 1 dF_dq, 2 the
 * diagonal Hessian blocks, 3 dF_dq_FD, 4 d2F_dq2_FD, 5 dF_dn); 9 outputs. */
int orc_term_eval(int term, int fn, int dir, int ns, const double *q, const double *x,
                  const int *spc, double *out);
/* The 5th-degree rule over the pair measure of a pair term (mode 0 F, 1
 * dF_dq, 2 d2F_dq2 of direction); 9 outputs. */
int orc_quad5(int term, int mode, int direction, const double *q, const double *sigma,
              const double *x, const int *spc, double *out);

/* Literal per-site drivers over a system of n sites (real + ghost) with CSR
 * neighbour lists for every site. */
void orc_mf_rho(int n, const double *q, const double *sigma, const double *x,
                const int *spc, const int *offs, const int *idx,
                const int *sites, int nsites, double *out);
void orc_V0(int n, const double *q, const double *sigma, const double *x,
            const int *spc, const double *rho, const int *offs,
            const int *idx, const int *sites, int nsites, double *out);
void orc_S0(int n, const double *q, const double *sigma, const double *x,
            const int *spc, const double *rho, const double *beta,
            const double *gamma, const int *offs, const int *idx,
            const int *sites, int nsites, double *out);
void orc_DV0_pairs(int n, const double *q, const double *sigma,
                   const double *x, const int *spc, const double *rho,
                   const int *offs, const int *idx, const int *u_list,
                   const int *i_list, int npairs, double *out4, double *out_x);
void orc_rho_nmf(int n, const double *q, const double *x, const int *spc,
                 const int *offs, const int *idx, const int *sites, int nsites,
                 double *out);

/* Non-mean-field forms (sigma -> 0), restated from MgHx-mf-V-bulk.cpp:
 * orc_pt_DV_pairs: dV_i/dq_u per (u, i) pair, 3 values
 *   (evaluate_DV_i_Dq_u_adp_MgHx, 147-330);
 * orc_pt_DV_dF: dV_i/dF per site, 9 values row-major, with reference
 *   positions q0 of every site (evaluate_DV_i_dF_MgHx, 530-704).
 * rho: the non-mean-field density of every site (orc_rho_nmf). */
void orc_pt_DV_pairs(int n, const double *q, const double *x, const int *spc,
                     const double *rho, const int *offs, const int *idx, const int *u_list,
                     const int *i_list, int npairs, double *out3);
void orc_pt_DV_dF(int n, const double *q, const double *q0, const double *x, const int *spc,
                  const double *rho, const int *offs, const int *idx, const int *sites,
                  int nsites, double *out9);

/* Non-mean-field d2V_i/dq_u^2 per (u, i) pair, 9 values row-major, as
 * evaluate_D2V_i_Dq2_u_MgHx (MgHx-mf-V-bulk.cpp:333-528) forms it. */
void orc_pt_D2V_pairs(int n, const double *q, const double *x, const int *spc,
                      const double *rho, const int *offs, const int *idx, const int *u_list,
                      const int *i_list, int npairs, double *out9);

/* Mean-field d2V0_i/dmean_q_u^2 per (u, i) pair, 9 values row-major
 * (evaluate_D2V0_i_Dmeanq2_u_MgHx, MgHx-mf-V-bulk.cpp:1366-1600); rho: the
 * mean-field density of every site. */
void orc_mf_D2V0_pairs(int n, const double *q, const double *sigma, const double *x,
                       const int *spc, const double *rho, const int *offs, const int *idx,
                       const int *u_list, const int *i_list, int npairs, double *out9);

/* Mean-field stretch derivative dV0_i/dF per site, 9 values row-major,
 * with reference positions q0 of every site (evaluate_DV0_i_dF_bulk_MgHx,
 * MgHx-mf-V-bulk.cpp:2329-2552); rho: the mean-field density of every site. */
void orc_mf_DV0_dF(int n, const double *q, const double *q0, const double *sigma,
                   const double *x, const int *spc, const double *rho, const int *offs,
                   const int *idx, const int *sites, int nsites, double *out9);

/* Residual assembly for real sites u (project definition):
 *   R_q(u)     = sum_{i in {u} U N(u)} (beta_i/beta_u) dV0_i/dq_u
 *   R_sigma(u) = sum_i (beta_i/beta_u) dV0_i/dsigma_u - 3/(beta_u sigma_u)
 *   R_x(u)     = sum_i (beta_i/beta_u) dV0_i/dx_u
 *                - (3/(2 x_u) + [x_u<1]/(1-x_u))/beta_u
 *                - [H and x_u<0.9999] gamma_u/beta_u           (H sites)
 * i.e. (1/beta_u) d(sum_i S0_i)/d(.)_u with S0 of MgHx-mf-V-bulk.cpp:957-1142.
 * Ghost centres use their owner's frame (owner/image arrays from
 * orc_ghosts; real sites have owner = self, image = 0).  Sites with
 * x_u < min_occupancy get zero residuals.  rho must hold every site's
 * mean-field density (ghosts: the owner's). */
void orc_residuals(int n, const double *q, const double *sigma,
                   const double *x, const int *spc, const double *beta,
                   const double *gamma, const double *rho, const int *owner,
                   const int *image, const int *offs, const int *idx,
                   const int *u_list, int nu, double *Rq, double *Rs,
                   double *Rx);

/* One hydrogen master-equation update (project definition, see
 * include/btam.h btam_dmd_step) on real sites: X holds the occupancy quanta
 * (2^-50) of the n real sites and is updated in place; mu the chemical
 * potentials; x_all/code_all/owner the all-sites occupancy, species code
 * (0 Mg, 1 H) and owner; moffs/midx the mechanical neighbours and
 * doffs/didx the diffusive neighbours of the real sites; params as
 * btam_dmd_step (dt, Df, dr, min_dx, max_x).  clipped (may be NULL) counts
 * the edge moves cut to a nonzero room. */
void orc_dmd_update(int n, const int *code_all, const int *owner, const double *x_all,
                    const double *beta, const double *mu, const int *moffs,
                    const int *midx, const int *doffs, const int *didx,
                    const double *params, long long *X, long long *clipped);
/* The step-control decision of btam_dmd_step_ctl for a step of params[0]
 * at the quanta X (same arguments as orc_dmd_update): out2[0] the largest
 * edge move over its nonzero room, out2[1] the largest site change over
 * max_dx (project definition). */
void orc_dmd_control(int n, const int *code_all, const int *owner, const double *x_all,
                     const double *beta, const double *mu, const int *moffs, const int *midx,
                     const int *doffs, const int *didx, const double *params, double max_dx,
                     const long long *X, double *out2);

#ifdef __cplusplus
}
#endif
#endif
