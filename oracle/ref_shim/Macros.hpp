// Build shim (test infrastructure only): stands in for the reference's
// src/Macros.hpp so that the reference's own arithmetic files
//   src/ADP/MgHx-ADP.cpp, src/ADP/MgHx-mf-V-bulk.cpp, src/ADP/density.cpp,
//   src/Numerical/cubic-spline.cpp, src/Numerical/Quadrature-Hermitian-3th.cpp,
//   src/Numerical/Quadrature-Measure.cpp
// compile unmodified without PETSc, MPI or Eigen.  It declares only the types,
// constants and helper macros those files use (Macros.hpp:29-42, 56-175,
// 238-329, 486-798, 803-881 of the reference).  Differences from the
// reference header, on purpose:
//   * DSQR is a thread-safe inline function (the reference writes a
//     file-static temporary, Macros.hpp:880-881, which races under OpenMP);
//   * PETSc scalar/index types are plain C types;
//   * the AtomicSpecie enum lists elements up to Cu only (ordinals match the
//     reference: XX = 0, H = 1, Mg = 12, Al = 13, Cu = 29).
#ifndef BTAM_REF_SHIM_MACROS_HPP
#define BTAM_REF_SHIM_MACROS_HPP

#include <Eigen/Dense>
#include <cmath>
#include <iostream>

typedef int PetscInt;
typedef int PetscMPIInt;
typedef int PetscErrorCode;
typedef double PetscScalar;
typedef double PetscReal;

#define PETSC_SUCCESS 0
#define PETSC_ERR_NOT_CONVERGED 91
#define PETSC_ERR_RETURN 99

#define sqrt_2 1.4142135623730951
#define sqrt_3 1.7320508075688772
#define sqrt_6 2.449489742783178

enum AtomicSpecie {
  XX, H, He, Li, Be, B, C, N, O, F, Ne, Na, Mg, Al, Si, P, S, Cl, Ar, K, Ca,
  Sc, Ti, V, Cr, Mn, Fe, Co, Ni, Cu
};

typedef struct {
  int numneigh;
  const PetscInt *mech_neighs_ptr;
} AtomTopology;

typedef struct {
  void (*F)(double *F, const double *xi, const double *q,
            const AtomicSpecie *spc);
  void (*dF_dq)(int direction, double *dF_dq, const double *xi,
                const double *q, const AtomicSpecie *spc);
  void (*d2F_dq2)(int direction, double *d2F_dq2, const double *xi,
                  const double *q, const AtomicSpecie *spc);
  void (*dF_dq_FD)(int direction, double *dF_dq, const double *xi,
                   const double *q, const AtomicSpecie *spc);
  void (*d2F_dq2_FD)(int direction, double *d2F_dq2, const double *xi,
                     const double *q, const AtomicSpecie *spc);
  void (*dF_dn)(int direction, double *dF_dn, const double *xi,
                const double *q, const AtomicSpecie *spc);
} potential_function;

typedef struct CubicSpline {
  double dx;
  int n;
  double *x;
  double *a, *b, *c, *d;
  double *db, *dc, *dd;
  double *ddc, *ddd;
} CubicSpline;

typedef struct adpPotential {
  int n_embed;
  int n_rho;
  int n_pair;
  int n_u;
  int n_w;
  CubicSpline embed;
  CubicSpline rho;
  CubicSpline pair;
  CubicSpline u;
  CubicSpline w;
  double mass;
  double radius;
  double factor;
  double r_cutoff;
} adpPotential;

// Function-pointer table of the mean-field equations (signatures as the
// reference's dmd_equations, Macros.hpp:540-798).
typedef struct dmd_equations {
  double (*evaluate_rho_i)(unsigned int, const Eigen::MatrixXd &,
                           const Eigen::VectorXd &, const AtomicSpecie *,
                           const AtomTopology);
  Eigen::Vector3d (*evaluate_DV_i_Dq_j)(unsigned int, unsigned int,
                                        const Eigen::MatrixXd &,
                                        const Eigen::VectorXd &,
                                        const Eigen::VectorXd &,
                                        const AtomicSpecie *,
                                        const AtomTopology);
  Eigen::Matrix3d (*evaluate_D2V_i_Dq2_j)(unsigned int, unsigned int,
                                          const Eigen::MatrixXd &,
                                          const Eigen::VectorXd &,
                                          const Eigen::VectorXd &,
                                          const AtomicSpecie *,
                                          const AtomTopology);
  Eigen::Matrix3d (*evaluate_DV_i_DF)(unsigned int, const Eigen::MatrixXd &,
                                      const Eigen::MatrixXd &,
                                      const Eigen::VectorXd &,
                                      const Eigen::VectorXd &,
                                      const AtomicSpecie *,
                                      const AtomTopology);
  double (*evaluate_mf_rho_i)(unsigned int, const Eigen::MatrixXd &,
                              const Eigen::VectorXd &,
                              const Eigen::VectorXd &, const AtomicSpecie *,
                              const AtomTopology);
  double (*evaluate_V0_i)(unsigned int, const Eigen::MatrixXd &,
                          const Eigen::VectorXd &, const Eigen::VectorXd &,
                          const Eigen::VectorXd &, const AtomicSpecie *,
                          const AtomTopology);
  double (*evaluate_S0_i)(unsigned int, const Eigen::MatrixXd &,
                          const Eigen::VectorXd &, const Eigen::VectorXd &,
                          const Eigen::VectorXd &, const Eigen::VectorXd &,
                          const Eigen::VectorXd &, const AtomicSpecie *,
                          const AtomTopology);
  Eigen::Vector3d (*evaluate_DV0_i_Dmeanq_j)(
      unsigned int, unsigned int, const Eigen::MatrixXd &,
      const Eigen::VectorXd &, const Eigen::VectorXd &,
      const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology);
  Eigen::Matrix3d (*evaluate_D2V0_i_Dmeanq2_j)(
      unsigned int, unsigned int, const Eigen::MatrixXd &,
      const Eigen::VectorXd &, const Eigen::VectorXd &,
      const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology);
  double (*evaluate_DV0_i_Dstdvq_j)(unsigned int, unsigned int,
                                    const Eigen::MatrixXd &,
                                    const Eigen::VectorXd &,
                                    const Eigen::VectorXd &,
                                    const Eigen::VectorXd &,
                                    const AtomicSpecie *, const AtomTopology);
  Eigen::Vector4d (*evaluate_DV0_i_Dq_j)(
      unsigned int, unsigned int, const Eigen::MatrixXd &,
      const Eigen::VectorXd &, const Eigen::VectorXd &,
      const Eigen::VectorXd &, const AtomicSpecie *, const AtomTopology);
  double (*evaluate_DV0_i_Dxi_j)(unsigned int, unsigned int,
                                 const Eigen::MatrixXd &,
                                 const Eigen::VectorXd &,
                                 const Eigen::VectorXd &,
                                 const Eigen::VectorXd &,
                                 const AtomicSpecie *, const AtomTopology);
  Eigen::Matrix3d (*evaluate_DV0_i_DF)(unsigned int, const Eigen::MatrixXd &,
                                       const Eigen::MatrixXd &,
                                       const Eigen::VectorXd &,
                                       const Eigen::VectorXd &,
                                       const Eigen::VectorXd &,
                                       const AtomicSpecie *,
                                       const AtomTopology);
} dmd_equations;

#define RESET "\033[0m"
#define RED "\033[31m"
#define GREEN "\033[32m"
#define YELLOW "\033[33m"

#define MAXW 100
#define MAXC 1000
#define NumberDimensions 3
#define TOL_NR 10E-6
#define TOL_zero 10E-23
#define PI 3.14159265358979323846

#define h_planck 6.5821192815E-4
#define k_B 8.617332478E-5
#define unit_change_uma 103.4993333E-6
#define unit_change_w 98.227002603

#define r_cutoff_ADP_MgHx 6.2934034034
#define r_cutoff_Eb 2.6
#define maxneigh 250
#define max_chemical_neighs 50

#define max_occupancy 0.99
#define min_occupancy 5e-4
#define min_stdv_q 0.001
#define max_stdv_q 3.0

static inline double btam_shim_dsqr(double a) { return a == 0.0 ? 0.0 : a * a; }
#define DSQR(a) btam_shim_dsqr(a)

#endif
