/* btam.h -- C ABI of the B200 mean-field ADP library (libbtam.so).
 *
 * A drop-in for the hot path of BT-AM's mean-field diffusive molecular
 * dynamics: the Gauss-Hermite-averaged angular-dependent potential (ADP) of
 * Mg-H over mean positions q, Gaussian widths sigma and occupancies x.  Each
 * entry point names the reference interface it replaces.  All functions take
 * caller-owned plain pointers (host unless the name says _device), return an
 * int status (BTAM_OK = 0), and never take ownership of caller memory.
 *
 * Units and encodings follow the reference: Angstrom, eV, ps; species are
 * atomic numbers (H = 1, Mg = 12) as in AtomicSpecie (src/Macros.hpp:56-175);
 * positions are row-major N x 3 doubles (the DMSwarm coordinate field).
 *
 * Threading: distinct systems may be used from distinct host threads; one
 * system must not be used by two threads at once.  Every system owns one
 * CUDA stream; work on different systems overlaps on the device.
 */
#ifndef BTAM_H
#define BTAM_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------
 * The reference's set-up functions return PetscErrorCode (0 or 99,
 * src/Macros.hpp:29-38); its evaluators have no error channel. */
#define BTAM_OK 0
#define BTAM_ERR_ARG 1               /* bad argument / null pointer */
#define BTAM_ERR_IO 2                /* table file missing or malformed (init_adp_MgHx returns EXIT_FAILURE, MgHx-ADP.cpp:389-392) */
#define BTAM_ERR_NEIGHBOR_OVERFLOW 3 /* > maxneigh = 250 neighbours (Neighbors.cpp:96-104) */
#define BTAM_ERR_NO_NEIGHBORS 4      /* a site without neighbours (Neighbors.cpp:106-113) */
#define BTAM_ERR_BOX_TOO_SMALL 5     /* periodic cell thinner than 2 rc (Atom.cpp:230-255) */
#define BTAM_ERR_NONFINITE 6         /* NaN/Inf in an input or output */
#define BTAM_ERR_OOM 7               /* device allocation failed */
#define BTAM_ERR_CUDA 8              /* other CUDA runtime error */
#define BTAM_ERR_GHOST_OVERFLOW 9    /* periodic images exceed capacity */
#define BTAM_ERR_OCCUPANCY 10        /* non-H site with 0 < x < min_occupancy (unsupported) */
#define BTAM_ERR_SPECIES 11          /* species other than H (1) or Mg (12) */
#define BTAM_ERR_TIMEOUT 12          /* a bounded device wait gave up */
#define BTAM_ERR_NOT_BUILT 13        /* neighbour lists not built yet */
#define BTAM_ERR_OUT_OF_BOX 14       /* site outside the cell along a periodic axis */
#define BTAM_ERR_TOO_LARGE 15        /* more sites than btam_mf_eval_noalloc's static scratch holds,
                                        or a batch beyond 32-bit site / pair indices */

/* arithmetic forms */
#define BTAM_FP64 0   /* plain FP64 drop-in */
#define BTAM_FP32C 1  /* FP32 quadrature/splines, compensated accumulation, FP64 reductions */

/* table ids for btam_tables_spline */
#define BTAM_T_RHO_MG 0
#define BTAM_T_RHO_H 1
#define BTAM_T_F_MG 2
#define BTAM_T_F_H 3
#define BTAM_T_PHI_MGMG 4
#define BTAM_T_PHI_HH 5
#define BTAM_T_PHI_MGH 6
#define BTAM_T_U_MGMG 7
#define BTAM_T_U_HH 8
#define BTAM_T_U_MGH 9
#define BTAM_T_W_MGMG 10
#define BTAM_T_W_HH 11
#define BTAM_T_W_MGH 12

/* reference constants (src/Macros.hpp:857-869) */
#define BTAM_R_CUTOFF 6.2934034034
#define BTAM_R_CUTOFF_EB 2.6          /* H-H diffusive pairs */
#define BTAM_MAXNEIGH 250
#define BTAM_MAX_CHEMICAL_NEIGHS 50
#define BTAM_MIN_OCCUPANCY 5e-4

/* relaxation schedules for btam_relax */
#define BTAM_RELAX_FP64 0        /* every evaluation in FP64 */
#define BTAM_RELAX_MIXED 1       /* FP32C until |R| < 1e-5, then FP64 */
#define BTAM_RELAX_FP32C 2       /* FP32C only (stops at its ~1e-6 noise floor) */
#define BTAM_RELAX_NEWTON 3      /* btam_relax_newton (FP64): max_iter Newton steps, m unused */
#define BTAM_RELAX_NGMRES 4      /* N-GMRES(m) with the critical-point line search (FP64): the
                                    reference's SNES options (main-BT-AM.cpp:64-67, m = 3) */

typedef struct btam_tables btam_tables;
typedef struct btam_system btam_system;
typedef struct btam_batch btam_batch;

const char *btam_status_string(int status);
int btam_version(void);
/* Name of the CUDA runtime error behind the calling thread's last
 * BTAM_ERR_CUDA or BTAM_ERR_OOM ("cudaErrorInvalidValue", ...; "" if none). */
const char *btam_last_cuda_error(void);
/* Bytes of the library's device-memory pool on the current device (no
 * counterpart in the reference): in use by live systems, batches and
 * servers, and reserved from the device.  Every device allocation of the
 * library comes from this pool, so a call that leaves both unchanged
 * allocated nothing that it kept. */
int btam_pool_usage(long long *used, long long *reserved);

/* Replaces init_adp_MgHx(&adp_MgMg, MgMg, dir), (&adp_HH, HH, dir),
 * (&adp_MgH, MgH, dir) (src/ADP/MgHx-ADP.cpp:366-501; called at
 * main-BT-AM.cpp:108-110): reads adpmg.dat, adph.dat and adpmgh.dat from
 * `dir` and uploads the splines to the current CUDA device. */
int btam_tables_load(const char *dir, btam_tables **out);
/* Replaces destroy_adp_MgHx (MgHx-ADP.cpp:505). */
void btam_tables_destroy(btam_tables *t);
/* Element mass of a species as read from the tables (element_mass[],
 * MgHx-ADP.cpp:436).  Returns 0 for unknown species. */
double btam_tables_mass(const btam_tables *t, int species);
/* Replaces cubic_spline / d_cubic_spline (src/Numerical/cubic-spline.cpp:
 * 84-112) on one table, evaluated on the device in FP64 for n host radii. */
int btam_tables_spline(const btam_tables *t, int table, int n, const double *r,
                       double *value, double *deriv);

/* The per-term plugin table (potential_function, Macros.hpp:252-278) of
 * the four ADP terms: term 0 rho_ij (MgHx-ADP.cpp:526-844), 1 V_pair_ij
 * (869-1209), 2 V_dipole_ij1j2 (1233-1758), 3 V_quadrupole_ij1j2
 * (1781-2434), for n geometries at once on the device, FP64.  fn selects
 * the slot: 0 F, 1 dF_dq, 2 d2F_dq2, 3 dF_dq_FD, 4 d2F_dq2_FD, 5 dF_dn;
 * direction is the slot's direction argument (a site for 1, 3 and 5; a
 * block ns * a + b for 2 and 4).  q: 9 per geometry (site-major, 6 used
 * by the pair terms), x and species: 3 per geometry (species 12 = Mg,
 * 1 = H; 2 used by the pair terms), out: 9 per geometry, the slot's
 * values first (1 for F and dF_dn, 3 for dF_dq, a 3x3 row-major block for
 * the Hessians) and zeros after.  Where the reference leaves a value
 * unset (the triplet Hessian blocks other than 0, 4, 5, 7 and 8, the
 * off-diagonal entries of the FD Hessians, the quadrupole's FD blocks other
 * than 0, 4 and 8) out holds 0, as the reference's zeroed outputs do.  The
 * finite-difference gradient steps by 1e-4, by 1e-5 for V_pair_ij, as the
 * reference's do.  BTAM_ERR_SPECIES for a species other
 * than 12 and 1. */
int btam_term_eval(const btam_tables *t, int term, int fn, int direction, int n,
                   const double *q, const double *x, const int *species, double *out);
/* The same terms averaged over the mean-field measure of each geometry
 * (means q, widths sigma: 3 per geometry) with the degree-3 rule:
 * mode 0 meanfield_integral_gh3th, 1 _gh_3th_dmq (d/d mean q of slot,
 * 3 values), 2 _gh3th_dsq (d/d sigma of slot), 3 _gh_3th_dxi (d/dx of
 * slot) (Quadrature-Hermitian-3th.cpp:36-378) over the pair or triplet
 * measure (Quadrature-Measure.cpp:30-109); coincident != 0 (triplets
 * only) is the measure with j1 = j2, one group for both.  out: 9 per
 * geometry, the 1 or 3 values first. */
int btam_term_quadrature(const btam_tables *t, int term, int mode, int slot, int coincident,
                         int n, const double *q, const double *sigma, const double *x,
                         const int *species, double *out);
/* The reference's 5th-degree rule over the pair measure
 * (Quadrature-Hermitian-5th.cpp:31-432: moment_1th_Vij_gaussian_measure_5th,
 * moment_1th_grad_f_ and moment_1th_hess_f_gaussian_measure_5th_6d) of a
 * pair term (0 rho_ij, 1 V_pair_ij) for n geometries: mode 0 the average of
 * F, 1 of dF_dq(direction), 2 of d2F_dq2(direction).  q: 9 per geometry (6
 * used), sigma, x, species: 3 per geometry (2 used); out: 9 per geometry,
 * the 1, 3 or 9 values first.  No caller in the reference selects this rule
 * (its integrator switch offers the degree-3 and multipole rules only). */
int btam_term_quadrature5(const btam_tables *t, int term, int mode, int direction, int n,
                          const double *q, const double *sigma, const double *x,
                          const int *species, double *out);

/* Replaces read_dump_information + init_DMD_simulation (dump-input.cpp:
 * 51-214, Atom.cpp:80-431): one system of n sites with its DMSwarm fields
 * (coordinates, "stdv-q", "molar-fraction", "specie", "beta", "gamma").
 * The cell is given by its origin and three lattice vectors (rows of
 * cell[9]); an orthogonal box [lo, hi) is origin = lo, cell = diag(hi - lo).
 * periodic[a] != 0 makes axis a periodic (dump "pp"; 0 = "ff").
 * beta/gamma may be NULL (beta = 1/(k_B 300 K), gamma = 0). */
int btam_system_create(const btam_tables *t, int n, const double *q,
                       const double *sigma, const double *x,
                       const int *species, const double *beta,
                       const double *gamma, const double origin[3],
                       const double cell[9], const int periodic[3],
                       btam_system **out);
void btam_system_destroy(btam_system *s);
/* Replaces the DMSwarmGetField/RestoreField round trip of q, sigma, x
 * (main-BT-AM.cpp:174-228): new state from host arrays (any may be NULL).
 * Periodic images follow their owners (DMSwarmMigrateGhostField,
 * Ghosts.cpp:861-892). */
int btam_system_set_state(btam_system *s, const double *q, const double *sigma,
                          const double *x);
/* Current state of the real sites (after relaxation or master-equation
 * steps), into host arrays; any may be NULL.  Replaces reading the DMSwarm
 * fields back with DMSwarmGetField. */
int btam_system_get_state(btam_system *s, double *q, double *sigma, double *x);
/* Sizes: real sites, periodic images, neighbour-list entries. */
int btam_system_info(const btam_system *s, int *n_real, int *n_ghost, long long *n_pairs);
/* The system's CUDA stream (cudaStream_t), for callers that time or order
 * work against it. */
void *btam_system_stream(const btam_system *s);

/* Replaces DMSwarmCreateGhostAtoms (Ghosts.cpp:42-802) +
 * list_of_active_mechanical_sites_MgHx (Topology.cpp:53-132) + neighbors
 * (Neighbors.cpp:39-134).  all_sites = 1 builds lists for images too, as the
 * reference does; 0 builds them for real sites only (what evaluation needs). */
int btam_neighbors_build(btam_system *s, int all_sites);
/* Copies the CSR lists (ascending neighbour index, images numbered after the
 * real sites).  offs holds n_list + 1 entries; idx_cap bounds idx. */
int btam_neighbors_copy(const btam_system *s, int *offs, int *idx, long long idx_cap);
/* Copies the periodic images: positions (n_ghost x 3), owning real site and
 * integer image shift (image = q_ghost - q_owner in lattice vectors). */
int btam_ghosts_copy(const btam_system *s, double *q, int *owner, int *image);

/* Replaces the per-site loop of evaluate_mf_rho_i_adp_MgHx
 * (MgHx-mf-V-bulk.cpp:708-787) over all real sites. */
int btam_mf_rho(btam_system *s, int precision, double *rho);

/* One residual evaluation of every real site.  Replaces the per-site loops
 * over evaluate_mf_rho_i_adp_MgHx, evaluate_V0_i_adp_MgHx (791-953),
 * evaluate_S0_i_adp_MgHx (957-1142), evaluate_DV0_i_Dq_u_MgHx (1823-2098) and
 * evaluate_DV0_i_Dxi_u_adp_MgHx (2102-2325), assembled as
 *   R_q(u) = sum_{i in {u} U N(u)} (beta_i/beta_u) dV0_i/dq_u
 *   R_sigma(u) = sum_i (beta_i/beta_u) dV0_i/dsigma_u - 3/(beta_u sigma_u)
 *   R_x(u) = sum_i (beta_i/beta_u) dV0_i/dx_u - (3/(2x_u) + [x_u<1]/(1-x_u))/beta_u
 *            - [x_u<0.9999] gamma_u/beta_u        (H sites; 0 for Mg)
 * i.e. (1/beta_u) times the gradient of sum_i S0_i.  Any output may be NULL.
 * totals (4): sum V0, sum S0, sum |R_q|^2 + R_sigma^2, sum R_x^2. */
int btam_mf_eval(btam_system *s, int precision, double *rho, double *V0,
                 double *S0, double *Rq, double *Rs, double *Rx, double *totals);
/* btam_system_set_state followed by btam_mf_eval in one call that waits
 * for the device once (no counterpart in the reference): the new state (any
 * of q, sigma, x may be NULL) is copied, checked and applied on the device,
 * then evaluated.  A rejected state returns the set_state error and leaves
 * the system's state unchanged; the outputs then hold the evaluation of
 * that unchanged state. */
int btam_mf_eval_state(btam_system *s, int precision, const double *q, const double *sigma,
                       const double *x, double *rho, double *V0, double *S0, double *Rq,
                       double *Rs, double *Rx, double *totals);
/* btam_mf_eval_state without the wait (no counterpart in the reference):
 * enqueues the copy of the new state, its check and update, the evaluation
 * and the copies of the results, and returns a ticket.  The host copies run
 * on two copy streams of the system, so a call's results travel to the host
 * while the next call evaluates: with pinned host buffers, a stream of
 * states costs about the evaluations alone.  Two calls may be in flight; a
 * third waits for the first to finish (its status is kept for its wait).
 * The host buffers of a call must stay untouched until its wait returns.
 * Other calls on the system are ordered after the evaluations but not after
 * the copies out: wait for every ticket first.  Not for systems of the job
 * server (BTAM_ERR_ARG). */
int btam_mf_eval_state_async(btam_system *s, int precision, const double *q,
                             const double *sigma, const double *x, double *rho, double *V0,
                             double *S0, double *Rq, double *Rs, double *Rx, double *totals,
                             long long *ticket);
/* Waits for the call of `ticket` to deliver its results; returns its status
 * (the statuses of btam_mf_eval_state).  BTAM_ERR_ARG for a ticket unknown
 * or already waited for. */
int btam_mf_eval_state_wait(btam_system *s, long long ticket);
/* The same evaluation enqueued on the system's stream with inputs and
 * outputs resident on the device; results stay in the system's buffers
 * (btam_results_copy reads them).  Does not synchronise. */
int btam_mf_eval_async(btam_system *s, int precision);
/* The occupancy gradients alone, enqueued like btam_mf_eval_async: rho-bar,
 * V0, S0 and R_x of the state (rho-bar, V0, S0 bit for bit the full
 * evaluation's, R_x to its last bits: a multiply-add of the shared
 * expressions may fuse differently without the derivative terms), with
 * R_q and R_sigma written as 0; evaluate_DV0_i_Dxi_u_adp_MgHx
 * (MgHx-mf-V-bulk.cpp:2102-2325) assembled as in btam_mf_eval.  These are
 * the master equation's chemical potentials; btam_dmd_step takes them this
 * way and keeps the pair rule's position-only sums between its steps.  The
 * directed kernel variants and a served job's evaluations compute the full
 * residuals instead. */
int btam_mf_eval_x(btam_system *s, int precision);
int btam_results_copy(btam_system *s, double *rho, double *V0, double *S0,
                      double *Rq, double *Rs, double *Rx, double *totals);
/* Waits for the system's stream and returns the first error it raised. */
int btam_system_sync(btam_system *s);
/* Autotuner (no counterpart in the reference): times every compiled block
 * shape / register cap of the two kernels, each with a full grid and with a
 * persistent grid of resident blocks, on this system and keeps the fastest
 * for later evaluations in `precision`; reports the chosen variant ids
 * (shape index, plus 8 for the persistent grid).  A given variant is bitwise
 * reproducible; the grid (full or persistent) never changes a bit, while
 * two block shapes are separate compilations and may round differently in
 * the last bits (within the stated tolerance of the form). */
int btam_autotune(btam_system *s, int precision, int *pass1_variant, int *pass2_variant);
/* Pins the launch variants of `precision` (as reported by btam_autotune),
 * for runs that must reproduce one another bit for bit. */
int btam_set_variants(btam_system *s, int precision, int pass1_variant, int pass2_variant);

/* Mean-field stress: W0 (9 per real site, row-major; row: gradient
 * component, column: position component) = dV0_u/dF at fixed sigma and x,
 * at reference positions q0 = q: evaluate_DV0_i_dF_bulk_MgHx
 * (MgHx-mf-V-bulk.cpp:2329-2552).  At reference positions q0 =
 * diag(F)^-1 q it is W0(a, b) / F_b.  total (9): the sum over the real
 * sites.  Runs the directed pass 1 first, so the system's rho, V0 and S0
 * buffers hold the current state's values afterwards.  Either output may
 * be NULL. */
int btam_mf_stress(btam_system *s, int precision, double *W0, double *total);

/* The per-pair terms of the residual assembly, unweighted, one value per
 * call of the reference's per-pair functions (the whole assembly that
 * btam_mf_eval returns is their beta-weighted sum):
 *   self (5 per real site u, may be NULL):  dV0_u/dq_u (3), dV0_u/dsigma_u,
 *        dV0_u/dx_u = evaluate_DV0_i_Dq_u_MgHx(u, u) (MgHx-mf-V-bulk.cpp:
 *        1823-2098; its dq part also evaluate_DV0_i_Dmeanq_u_MgHx, 1146-1362,
 *        and its dsigma part evaluate_DV0_i_Dstdvq_u_MgHx, 1603-1819) and
 *        evaluate_DV0_i_Dxi_u_adp_MgHx(u, u) (2102-2325);
 *   slot (5 per entry p of the real sites' neighbour lists, in the order of
 *        btam_neighbors_copy; slot_cap entries of 5 at least, may be NULL):
 *        for u's entry p with neighbour j, dV0_j/d(q_u, sigma_u, x_u) = the
 *        same functions at (u, j).  For a periodic image j it is the value
 *        of j's owner o at the image of u that neighbours o with the
 *        opposite shift (translation invariance), the pair the reference
 *        evaluates for that entry.
 * Values are 0 when u or j is empty (x < min_occupancy).  The dx part is
 * defined for every species (the assembly keeps it for H sites only).
 * Directed kernels, in `precision`; runs the directed pass 1 first (the
 * system's rho, V0, S0 buffers then hold the current state's values). */
int btam_mf_pair_terms(btam_system *s, int precision, double *self, double *slot,
                       long long slot_cap);

/* Mean-field Hessian blocks: H (9 per real site, row-major) = sum over
 * i in {u} U N(u) of evaluate_D2V0_i_Dmeanq2_u_MgHx(u, i)
 * (MgHx-mf-V-bulk.cpp:1366-1600), FP64, as the reference forms each term
 * (for a neighbour i the diagonal blocks of u's slots; for j1 = j2 = u
 * without their cross blocks).  A direct evaluation of the reference's
 * sums (about N_nb^2 x 18 term Hessians per site), not the moment form of
 * the evaluation kernels: no solver needs it on a hot path.  Runs the FP64
 * pass 1 first (the system's rho, V0, S0 buffers then hold the current
 * state's values). */
int btam_mf_hessian(btam_system *s, double *H);
/* The same blocks one pair at a time, as the reference returns them:
 * Hself (9 per real site, may be NULL) = evaluate_D2V0_i_Dmeanq2_u_MgHx(u, u)
 * and Hslot (9 per entry of the real sites' lists, slot_cap entries at
 * least, may be NULL) = the block of the entry's neighbour i, (u, i). */
int btam_mf_hessian_pairs(btam_system *s, double *Hself, double *Hslot, long long slot_cap);

/* ---- the multipole rule (MULTIPOLE_INTEGRAL) ------------------------------
 * The reference's alternative mean-field rule behind its compile switch
 * (MgHx-mf-V-bulk.cpp:715-724; meanfield_integral_mp,
 * Quadrature-Multipole.cpp:97-143): <f> = f(mean) + sum over the measure's
 * dof table of sigma_a^2 / 2 tr d2f/dq_a dq_b.  Two Hessian variants:
 *   BTAM_MP_FD        as the reference's build flags compile it
 *                     (-DNUMERICAL_DERIVATIVES=0 satisfies the rule's
 *                     #ifdef): finite-difference Hessians, step 1e-4,
 *                     diagonal entries only (MgHx-ADP.cpp:736-812,
 *                     1091-1167, 1605-1680, 2270-2349);
 *   BTAM_MP_ANALYTIC  NUMERICAL_DERIVATIVES undefined: analytic Hessians.
 * Replaces evaluate_mf_rho_i_adp_MgHx (708-787), evaluate_V0_i_adp_MgHx
 * (791-953) and evaluate_S0_i_adp_MgHx (957-1142) built with that rule:
 * rho (n_real, may be NULL) the multipole rho-bar, V0 and S0 (n_real each,
 * may be NULL) per site, *energy (may be NULL) the sum of V0.  FP64, a
 * direct evaluation of the reference's pair and triplet sums on the
 * system's neighbour lists (kept as built). */
#define BTAM_MP_FD 1
#define BTAM_MP_ANALYTIC 2
int btam_mf_eval_multipole(btam_system *s, int rule, double *rho, double *V0, double *S0,
                           double *energy);
/* The residuals of every real site under the same rule: Rq (3 n_real), Rs
 * and Rx (n_real each), assembled as btam_mf_eval's.  The per-pair parts
 * replace evaluate_DV0_i_Dq_u_MgHx (1823-2098) built with the rule
 * (meanfield_integral_mp_dmq: the gradient plus sigma_s^2 / 2 times its
 * five-point second difference, step 0.01, in every coordinate of every
 * slot; meanfield_integral_mp_dsq: sigma times the Hessian traces) and
 * evaluate_DV0_i_Dxi_u_adp_MgHx (2102-2325), whose occupancy integrals the
 * reference keeps on the degree-3 rule, at the multipole rho-bar.  FP64,
 * a direct evaluation: one warp per (site, centre) pair. */
int btam_mf_residuals_multipole(btam_system *s, int rule, double *Rq, double *Rs,
                                double *Rx);
/* The mean-field stress under the same rule, as btam_mf_stress: W0 (9 per
 * real site, row-major) = evaluate_DV0_i_dF_bulk_MgHx (2329-2552) built
 * with the rule (its meanfield_integral_mp_dmq) at reference positions q0 =
 * q; total (9) their sum.  Either output may be NULL.  FP64, direct. */
int btam_mf_stress_multipole(btam_system *s, int rule, double *W0, double *total);
/* The mean-field Hessian blocks under the same rule, as btam_mf_hessian:
 * evaluate_D2V0_i_Dmeanq2_u_MgHx (1366-1600) built with the rule, which
 * takes its rho gradient from meanfield_integral_mp_dmq (1476) and keeps
 * the term blocks on the degree-3 rule (meanfield_integral_gh_3th_d2mq),
 * at the multipole rho-bar.  H: 9 per real site.  FP64. */
int btam_mf_hessian_multipole(btam_system *s, int rule, double *H);

/* The per-pair terms under the multipole rule, as btam_mf_pair_terms: self
 * (5 per real site) and slot (5 per list entry, slot_cap entries at least),
 * either may be NULL; evaluate_DV0_i_Dq_u_MgHx (1823-2098) and
 * evaluate_DV0_i_Dxi_u_adp_MgHx (2102-2325) built with the rule, FP64. */
int btam_mf_pair_terms_multipole(btam_system *s, int rule, double *self, double *slot,
                                 long long slot_cap);
/* Per-pair Hessian blocks: Hself (9 per real site) the block of i = u and
 * Hslot (9 per list entry, slot_cap entries at least) the block of the
 * entry's neighbour i, evaluate_D2V0_i_Dmeanq2_u_MgHx(u, u) and (u, i)
 * (1366-1600) built with the rule.  Both outputs are required. */
int btam_mf_hessian_pairs_multipole(btam_system *s, int rule, double *Hself, double *Hslot,
                                    long long slot_cap);

/* Replaces evaluate_rho_i_adp_MgHx_kokkos (src/ADP/density.cpp:44-104), the
 * non-mean-field density the shipped main-BT-AM.cpp evaluates (197-207). */
int btam_rho_nmf(btam_system *s, double *rho);

/* ---- non-mean-field forms (sigma -> 0: every term at the mean positions) --
 * One device evaluation over the system's neighbour lists (kept as built):
 *   rho (n): rho_i = sum_j x_j rho_{s_j}(|q_j - q_i|), as btam_rho_nmf
 *            (evaluate_rho_i_adp_MgHx, MgHx-mf-V-bulk.cpp:83-143);
 *   V (n):   the point energy x_i F(rho_i) + sum_j 1/2 x_i x_j phi + the
 *            dipole and quadrupole sums over j1 <= j2 (no reference function
 *            returns it; 0 for x_i < min_occupancy);
 *   Fq (3n): sum_{i in {u} U N(u)} dV_i/dq_u per real site u, the assembled
 *            evaluate_DV_i_Dq_u_adp_MgHx (147-330);
 *   W (9n):  dV_u/dF per real site, row-major (row: gradient component,
 *            column: position component), at reference positions q0 = q
 *            (evaluate_DV_i_dF_MgHx, 530-704).  At reference positions
 *            q0 = diag(F)^-1 q it is W(a, b) / F_b;
 *   totals (12): sum V, sum |Fq|^2, sum of W over the sites (9), 0.
 * Any output may be NULL.  sigma is not read. */
int btam_pt_eval(btam_system *s, double *rho, double *V, double *Fq, double *W,
                 double *totals);
/* Hessian blocks of the non-mean-field forms: H (9 per real site,
 * row-major) = sum_{i in {u} U N(u)} evaluate_D2V_i_Dq2_u_MgHx(u, i)
 * (MgHx-mf-V-bulk.cpp:333-528), as the reference forms each term: for
 * i = u the Hessian of V_u in q_u; for a neighbour i the diagonal blocks of
 * the slots u holds in V_i's terms (for j1 = j2 = u the two slot blocks
 * without their cross blocks, so this is not d2(sum V)/dq_u^2 there). */
int btam_pt_hessian(btam_system *s, double *H);
/* The non-mean-field gradient and Hessian terms one pair at a time, as the
 * reference's per-pair functions return them (any output may be NULL):
 *   self3 (3 per real site) = evaluate_DV_i_Dq_u_adp_MgHx(u, u) (147-330),
 *   slot3 (3 per entry of the real sites' lists) = the same at (u, i) for
 *         the entry's neighbour i,
 *   Hself (9 per real site) = evaluate_D2V_i_Dq2_u_MgHx(u, u) (333-528),
 *   Hslot (9 per entry) = the same at (u, i);
 * slot_cap bounds the entries of slot3 and Hslot. */
int btam_pt_pair_terms(btam_system *s, double *self3, double *slot3, double *Hself,
                       double *Hslot, long long slot_cap);
/* Stretches the system by diag(F) (F[a] > 0): q <- F q for every site, the
 * cell rows and the origin likewise; images follow; neighbour lists are
 * kept.  BTAM_ERR_BOX_TOO_SMALL (nothing changed) if a periodic cell would
 * become narrower than 2 rc. */
int btam_stretch_apply(btam_system *s, const double F[3]);
/* Bulk stretch relaxation: replaces mechanical_relaxation_bulk
 * (Mechanical-Relaxation-bulk.cpp:123-437), the reference's one compiled
 * solver.  Finds the diagonal stretch F with
 *   Y_a(F) = (1/V0) sum_u dV_u/dF(a, a) = 0,  q = diag(F) q_ref,
 * V0 = |det cell| at entry, dV_u/dF of the non-mean-field forms at fixed x
 * and fixed neighbour lists (evaluate_RHS, 441-600).  Newton's method with
 * the Jacobian by forward differences (three extra residuals per
 * iteration, as the reference's MatFDColoring of the dense 3x3 pattern) and
 * a backtracking line search on |Y|^2; converged when |Y| <= atol or
 * |Y| <= rtol |Y(F_start)| (the reference: 1e-12, 1e-10, at most 20
 * iterations).  F (3): the start on entry (the reference starts at 1), the
 * solution on return, and the system is left stretched by it (cell and
 * origin too, 366-384).  info (5, may be NULL): final |Y|, iterations,
 * residual evaluations, status (1 converged, 0 iteration limit, -1 no
 * descent), V0.  The reference's options select PETSc's NGMRES with a
 * critical-point line search (main-BT-AM.cpp:64-67); PETSc is not used
 * here, and any solver that converges finds the same F. */
int btam_relax_stretch(btam_system *s, double atol, double rtol, int max_iter, double F[3],
                       double *info);
/* The same relaxation with the solver the reference's main program
 * configures for it (main-BT-AM.cpp:64-67: -minV_dF_snes_type ngmres,
 * -minV_dF_snes_ngmres_m 3, -minV_dF_snes_linesearch_type cp): N-GMRES(m)
 * with the critical-point line search, PETSc SNESNGMRES's difference
 * selection and restart with their defaults; three residual evaluations per
 * iteration.  m = 1..3 (the stretch has three unknowns); info as
 * btam_relax_stretch. */
int btam_relax_stretch_ngmres(btam_system *s, int m, double atol, double rtol, int max_iter,
                              double F[3], double *info);
/* The same relaxation on the mean-field stress (btam_mf_stress: the
 * reference's evaluate_DV0_i_dF_bulk_MgHx, whose table slot
 * evaluate_DV0_i_DF no reference solver calls) at fixed sigma and x, in
 * `precision` (BTAM_FP64 or BTAM_FP32C; the FP32C stress resolves |Y| to
 * about 1e-9 eV/A^3, so give it atol >= 1e-8). */
int btam_relax_stretch_mf(btam_system *s, int precision, double atol, double rtol,
                          int max_iter, double F[3], double *info);

/* ---- consumers of the evaluation -----------------------------------------
 * Relaxation of (q, sigma).  The reference configures a PETSc SNES
 * (mechanical_relaxation_bulk, Mechanical-Relaxation-bulk.cpp:123-437; options
 * at main-BT-AM.cpp:64-67) but solves only a 3-stretch bulk problem; this
 * relaxes the q and sigma of every site with x >= x_min.  It minimises
 *   F = sum_i beta_i V0_i - 3 sum_u log sigma_u   over (q, log sigma),
 * whose gradient is beta_u (R_q(u), sigma_u R_sigma(u)), with sigma_min <=
 * sigma <= sigma_max, by L-BFGS (m pairs, 1 <= m <= 16) on occupancy-scaled
 * variables (sqrt(x) z) with an Armijo backtracking line search, on the
 * device, until the projected residual norm sqrt(sum |R_q|^2 + R_sigma^2)
 * over the relaxed sites (sigma components held at a bound excluded) is
 * <= tol, or max_iter iterations.  mode: BTAM_RELAX_*.  Neighbour lists stay
 * fixed, as in the reference.
 * bounds (3, NULL = defaults): sigma_min (0.001 A, min_stdv_q of
 * Macros.hpp:870), sigma_max (0.4 A: beyond ~0.43 A the 3-sigma quadrature
 * points of the closest H-H pair, 1.30 A apart, pass through r = 0; the
 * reference's max_stdv_q = 3.0 lets near-empty sites spread across their
 * neighbours), x_min (0.01: sites below it are held fixed, since their
 * energy scales with x and they barely resist moving).
 * info (5, may be NULL): final residual norm, iterations, evaluations, final
 * F, status (1 converged, 0 iteration limit, -1 no further decrease). */
int btam_relax(btam_system *s, int mode, double tol, int max_iter, int m,
               const double *bounds, double *info);

/* Newton option of the same relaxation (the reference's SNES is a Newton
 * method, NEWTONLS, Mechanical-Relaxation-bulk.cpp:293): damped truncated
 * Newton on the same F and variables, FP64.  Each step solves
 * (H + lam I) p = -g by conjugate gradients (at most max_cg iterations,
 * forcing term min(0.5, sqrt|g|)), with H d from a forward difference of
 * the gradient (one residual evaluation per CG iteration; no Hessian is
 * formed); negative curvature raises the damping lam and restarts the
 * solve, full steps lower it.  Then an Armijo backtracking line search (no
 * q or log sigma moves more than 0.2 per step).  Converged at the projected
 * residual norm <= tol, or max_newton steps.  bounds as btam_relax.
 * info (6, may be NULL): final norm, Newton steps, evaluations, final F,
 * status (1 converged, 0 step limit, -1 no further decrease), CG
 * iterations. */
int btam_relax_newton(btam_system *s, double tol, int max_newton, int max_cg,
                      const double *bounds, double *info);

/* Hydrogen master equation (absent from the reference, which keeps only its
 * parameters, Variables.hpp:68-92, and the diffusive graph builder
 * list_of_diffusive_neighs, Neighbors.cpp:139-275).  Setup builds the H-H
 * graph (pairs within 2.6 A, at most 50 per site) and carries every H
 * occupancy as an integer number of 2^-50 quanta from then on.  A step:
 * evaluates the occupancy gradients (btam_mf_eval_x; after the steps the
 * system's stored R_q and R_sigma are 0 until the next full evaluation),
 * forms the chemical potential
 *   mu_i = R_x(i) + [x_i<0.9999] gamma_i/beta_i     (x_i >= 5e-4)
 *   mu_i = -(3/(2x) + 1/(1-x))/beta_i, x = max(x_i, 1e-12)   (emptier sites)
 * of every H site that is diffusively active (x_i plus the x of its H
 * neighbours within r_c >= 0.01, Topology.cpp:202-364) and moves, across
 * every edge between active sites,
 *   dt * Df/dr^2 * (beta_i+beta_j)/2 * xm(1-xm) * (mu_i - mu_j),  xm = (x_i+x_j)/2,
 * rounded to quanta, skipped below min_dx, limited so that no site leaves
 * [0, max(max_x, x)], from i to j.  Total hydrogen is conserved exactly.
 * params (5, NULL = reference values): dt (4e-4), Df (0.045), dr (3.2),
 * min_dx (1e-8), max_x (0.9).  total_quanta (2, may be NULL): 128-bit total
 * of the quanta after the steps, as (high, low) 64-bit halves. */
int btam_dmd_setup(btam_system *s);
int btam_dmd_step(btam_system *s, int precision, int nsteps, const double *params,
                  long long *total_quanta);
/* The same steps with step control (no counterpart in the reference).
 * Every step of length dt first takes the chemical potentials at the
 * current occupancies and from them two ratios: the largest move of an
 * edge over the room the degree split leaves it (edges whose room is zero,
 * an empty giver or a full receiver, move nothing and do not count), and
 * the largest change of a site's occupancy over max_dx.  The step is then
 * taken as m = min(max_sub, max(1, ceil(the larger ratio))) sub-steps of
 * dt / m, each with fresh chemical potentials (the first reuses the
 * decision's): a sub-step is exactly one btam_dmd_step of dt / m.
 * params (7, NULL = defaults): dt, Df, dr, min_dx, max_x as btam_dmd_step,
 * then max_dx (0.05) and max_sub (64).  stats (4, may be NULL): sub-steps
 * taken, steps that were subdivided, edge moves still cut to their room
 * (possible when a step needs more than max_sub sub-steps or the chemical
 * potentials change within it), the largest ratio seen.  Synchronises once
 * per step to read the decision. */
int btam_dmd_step_ctl(btam_system *s, int precision, int nsteps, const double *params,
                      long long *total_quanta, double *stats);
/* A mean-field DMD run (no counterpart in the reference, which keeps only
 * the method's parameters): nsteps master-equation steps with step control
 * (btam_dmd_step_ctl, params as there) and, after every relax_every steps,
 * a relaxation of (q, sigma) at the new occupancies (btam_relax with
 * relax_mode, relax_tol, relax_max_iter, history 8 (N-GMRES: 3), default
 * bounds), so the mechanical state follows the occupancy; relax_every = 0
 * never relaxes.
 * Neighbour lists and the diffusive graph stay as built.  stats (6, may be
 * NULL): sub-steps, subdivided steps, cut edge moves, the largest ratio
 * (as btam_dmd_step_ctl), relaxations run, their residual evaluations. */
int btam_dmd_run(btam_system *s, int precision, int nsteps, const double *params,
                 int relax_every, int relax_mode, double relax_tol, int relax_max_iter,
                 long long *total_quanta, double *stats);
/* Edge moves cut to a nonzero room by every master-equation step since
 * btam_dmd_setup (btam_dmd_step and btam_dmd_step_ctl alike). */
int btam_dmd_clip_count(btam_system *s, long long *clipped);
/* Current occupancies (n_real), their quanta and the last chemical
 * potentials; any pointer may be NULL. */
int btam_dmd_occupancy(btam_system *s, double *x, long long *quanta, double *mu);
/* The diffusive graph as CSR over the real sites (images numbered after the
 * real sites). */
int btam_dmd_graph_copy(const btam_system *s, int *offs, int *idx, long long idx_cap);

/* ---- evaluation without device allocation -------------------------------
 * No counterpart in the reference.  For callers that must not call
 * cudaMalloc/cudaFree (their device memory belongs to another allocator, or
 * an allocation's implicit synchronisation is not acceptable): the same
 * residual evaluation as btam_mf_eval_async on caller-owned DEVICE buffers,
 * with the kernels' scratch in a fixed array inside the library instead of
 * per-system allocations.
 * Inputs (device): pos4 = (x, y, z, sigma) and xb = (x, beta) per site,
 * code (0 = Mg, 1 = H) and owner (real site of each row) per site, real sites
 * first then periodic images; gamma per real site; offs/idx = neighbour CSR
 * of the real sites in that all-sites numbering.  Outputs (device): V0, Rs,
 * Rx per real site, Rq 3 per real site, totals[4] as btam_mf_eval.
 * Limit: n_real <= 16384 (BTAM_ERR_TOO_LARGE beyond).  The scratch (~10.9 MB
 * per device) lives until the process exits and is shared by every call on
 * that device: calls that overlap on the GPU race; serialise them.  Runs
 * on `stream` (a cudaStream_t, NULL = default); before returning it reads
 * the kernels' error flag back to the host and waits for `stream`, so the
 * host blocks until the evaluation has finished, and the call can never be
 * recorded into a CUDA graph (stream capture). */
int btam_mf_eval_noalloc(const btam_tables *t, int precision, int n_real,
                         const double *pos4, const double *xb, const int *code,
                         const int *owner, const double *gamma, const int *offs,
                         const int *idx, double *V0, double *Rq, double *Rs,
                         double *Rx, double *totals, void *stream);

/* ---- batched evaluation (no counterpart in the reference, which evaluates
 * one DMSwarm per process) -----------------------------------------------
 * A batch gathers many built systems (same tables, same device) into one
 * device layout: every system's real sites, then every system's images,
 * neighbour lists renumbered accordingly.  One evaluation of all systems is
 * a single CUDA graph (pass 1, pass 2, per-system totals) on the batch's own
 * stream, with persistent grids of resident blocks by default.  Each
 * system's results equal those of btam_mf_eval on the system alone, bitwise,
 * when both use the same block shapes (btam_set_variants /
 * btam_batch_set_variants).
 * The systems must outlive the batch; the batch keeps its own copy of their
 * state, refreshed by btam_batch_set_state. */
int btam_batch_create(btam_system *const *systems, int n_sys, btam_batch **out);
int btam_batch_destroy(btam_batch *b);
int btam_batch_info(const btam_batch *b, int *n_sys, int *n_real, int *n_all,
                    long long *n_pairs);
void *btam_batch_stream(const btam_batch *b);
/* New (q, sigma, x) of system k (NULL keeps a field), as
 * btam_system_set_state on that system, then copied into the batch. */
int btam_batch_set_state(btam_batch *b, int k, const double *q, const double *sigma,
                         const double *x);
/* Times every pass-1 / pass-2 launch variant (block shape; full or
 * persistent grid) on the whole batch and keeps the fastest. */
int btam_batch_autotune(btam_batch *b, int precision, int *pass1_variant, int *pass2_variant);
int btam_batch_set_variants(btam_batch *b, int precision, int pass1_variant, int pass2_variant);
/* Enqueues one evaluation of every system (one graph launch); does not
 * synchronise.  btam_batch_sync waits and returns the first error raised. */
int btam_batch_eval_async(btam_batch *b, int precision);
int btam_batch_sync(btam_batch *b);
/* Results of system k as btam_results_copy (NULL skips a field; totals[4]);
 * synchronises the batch's stream. */
int btam_batch_results_copy(btam_batch *b, int k, double *rho, double *V0, double *S0,
                            double *Rq, double *Rs, double *Rx, double *totals);
/* totals[4 k + c] of every system k; synchronises. */
int btam_batch_totals_copy(btam_batch *b, double *totals);

/* ---- job server (no counterpart in the reference, which runs one
 * simulation per MPI job) ---------------------------------------------------
 * Serves relaxation / master-equation / single-evaluation jobs of any size
 * concurrently on the current device.  Submission copies the job's inputs;
 * a job is admitted when a worker is free and its estimated device footprint
 * (btam_estimate_bytes) fits the memory budget next to the running jobs (a
 * job may overtake the head of the queue only if it leaves room for the
 * head).  Each running job owns a system and its stream: its state and
 * neighbour lists stay resident on the device until it ends.  Continuous
 * batching: the residual evaluations of the running jobs of up to 8192
 * sites are merged, round by round, into one batched evaluation (one set of
 * launches over those jobs' sites); jobs join at the next round after they
 * start and leave when they end.  Larger jobs run their own kernels on
 * their own streams, overlapping with the rounds.  A job's results equal those of the same job run alone
 * (deterministic kernels, fixed kernel shapes, rows never shared). */
typedef struct btam_server btam_server;

#define BTAM_JOB_RELAX 0  /* btam_relax(mode, tol, max_iter, lbfgs_m, bounds) */
#define BTAM_JOB_DMD 1    /* btam_dmd_setup + btam_dmd_step(precision, nsteps, dmd_params) */
#define BTAM_JOB_EVAL 2   /* one btam_mf_eval(precision) */
#define BTAM_JOB_STRETCH 3  /* btam_relax_stretch(atol = tol (0: 1e-12), rtol 1e-10,
                              max_iter (0: 20)) from F = 1; result: norm |Y|,
                              objective det F, iterations, evaluations,
                              converged; the final state is the stretched q */

typedef struct btam_job_spec {
  int kind;        /* BTAM_JOB_* */
  int precision;   /* BTAM_FP64 / BTAM_FP32C (DMD and EVAL jobs) */
  int mode;        /* BTAM_RELAX_* (relaxation jobs) */
  int n;           /* sites */
  const double *q, *sigma, *x;  /* as btam_system_create */
  const int *species;
  const double *beta, *gamma;   /* may be NULL */
  const double *origin, *cell;  /* [3], [9] */
  const int *periodic;          /* [3] */
  double tol;                   /* relaxation tolerance */
  int max_iter, lbfgs_m;        /* relaxation iterations, history m (0: 8; N-GMRES 3) */
  double sigma_min, sigma_max, x_min;  /* relaxation bounds (0: defaults) */
  int nsteps;                   /* master-equation steps */
  double dmd_params[5];         /* dt, Df, dr, min_dx, max_x */
  int plain;  /* 0: the server's kernels (undirected, persistent); nonzero:
                 the plain two-pass kernel pair (launch variants (0, 0)) */
} btam_job_spec;

typedef struct btam_job_result {
  int status;      /* BTAM_OK or the first error of the job */
  int kind;
  double t_submit, t_admit, t_start, t_end;  /* seconds since server creation */
  double norm;      /* relaxation: final projected residual norm; EVAL: sum R^2 */
  double objective; /* relaxation objective; EVAL: sum V0 */
  int iterations, evaluations, converged;
  long long h_quanta_hi, h_quanta_lo;  /* DMD: total H quanta (signed 128-bit) */
} btam_job_result;

/* Device bytes a job of n sites in this cell is admitted against. */
long long btam_estimate_bytes(int n, const double cell[9], const int periodic[3]);
/* n_workers concurrent jobs; budget_bytes <= 0 takes 80% of the free memory. */
int btam_server_create(const btam_tables *t, int n_workers, long long budget_bytes,
                       btam_server **out);
/* Queues a job; BTAM_ERR_TOO_LARGE if it can never fit the budget. */
int btam_server_submit(btam_server *srv, const btam_job_spec *spec, long long *job_id);
/* Waits (timeout_s < 0: forever; BTAM_ERR_TIMEOUT when it runs out) for a
 * job, returns its status and copies its result and final state (any pointer
 * may be NULL).  A result is collected once. */
int btam_server_wait(btam_server *srv, long long job_id, double timeout_s,
                     btam_job_result *result, double *q, double *sigma, double *x);
int btam_server_stats(btam_server *srv, long long *waiting, int *running,
                      long long *completed, long long *failed, long long *bytes_in_use);
/* Lets running jobs finish, drops the jobs still queued, joins the workers. */
int btam_server_destroy(btam_server *srv);
/* Continuous batching counters: evaluation rounds run, job evaluations
 * they served (each round serves every running job that asked), and
 * rebuilds of the shared batch layout (when jobs joined or left). */
int btam_server_batch_stats(btam_server *srv, long long *rounds, long long *evaluations,
                            long long *rebuilds);

/* ---- measurement (no counterpart in the reference, which has only PETSc's
 * SNES monitor for tracing) ------------------------------------------------ */
/* One evaluation as btam_mf_eval_async, with CUDA events on the system's
 * stream around each kernel: ms[0] the pass-1 pair-rule kernel, ms[1] the
 * pass-1 site kernel, ms[2] the pass-2 pair kernel, ms[3] the pass-2 site
 * kernel, ms[4] the totals (ms[0] and ms[2] are ~0 for the directed
 * variants, which have no pair kernels).  Synchronises. */
int btam_mf_eval_profile(btam_system *s, int precision, double ms[5]);
/* Sustained FMA throughput of the current device in TFLOP/s (FMA = 2 flops)
 * for fp64 = 0 (FP32) or 1 (FP64), from a register-resident FMA loop over
 * every SM lasting about `seconds`. */
int btam_probe_fma_peak(int fp64, double seconds, double *tflops);
/* Device-wide throughput (GB/s) of random 32-byte record gathers from the
 * FP32 radial tables (L1-resident), the access pattern of the evaluation
 * kernels' quadrature points; one launch timed after calibration to about
 * `seconds`. */
int btam_probe_gather_peak(const btam_tables *t, double seconds, double *gbs);

#ifdef __cplusplus
}
#endif
#endif /* BTAM_H */
