// Test infrastructure only: the CPU oracle (see btam_oracle.h).
//
// A literal restatement of the reference's arithmetic for the mean-field ADP
// path.  Every function names the reference file:line it follows.  It keeps
// the reference's loop structure (pair loop, j1 <= j2 triplet loop, one
// Gaussian measure per pair/triplet) and its occupancy-threshold quirks; it
// only replaces the per-call heap allocations with stack arrays and the Eigen
// temporaries with plain arrays, which does not change any arithmetic.
// Build: oracle/Makefile (-O2 -ffp-contract=off, IEEE double).
#include "btam_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

namespace {

// Constants of the reference (Macros.hpp:40-42, 846-871).
const double kSqrt2 = 1.4142135623730951;
const double kMinOcc = 5e-4;           // min_occupancy
const double kHbar = 6.5821192815E-4;  // h_planck [eV ps]
const double kUma = 103.4993333E-6;    // unit_change_uma
const int kH = 1, kMg = 12;            // AtomicSpecie ordinals
const int kErrNeighborOverflow = 3, kErrNoNeighbors = 4, kErrBoxTooSmall = 5,
          kErrGhostOverflow = 9;

// ---------------------------------------------------------------------------
// Cubic splines (Macros.hpp:286-329; cubic-spline.cpp:84-128)
struct Spline {
  double dx = 0;
  int n = 0;
  std::vector<double> a, b, c, d, db, dc, dd, ddc, ddd;
};

double spline_val(const Spline &s, double x) {
  int m = static_cast<int>(x / s.dx);
  m = std::min(m, s.n - 1);
  double p = m * s.dx;
  p = x - p;
  p = std::min(p, s.dx);
  return s.a[m] + (s.b[m] + (s.c[m] + s.d[m] * p) * p) * p;
}
double spline_d1(const Spline &s, double x) {
  int m = static_cast<int>(x / s.dx);
  m = std::min(m, s.n - 1);
  double p = m * s.dx;
  p = x - p;
  p = std::min(p, s.dx);
  return s.db[m] + (s.dc[m] + s.dd[m] * p) * p;
}
double spline_d2(const Spline &s, double x) {
  int m = static_cast<int>(x / s.dx);
  m = std::min(m, s.n - 1);
  double p = m * s.dx;
  p = x - p;
  p = std::min(p, s.dx);
  return s.ddc[m] + s.ddd[m] * p;
}

// adpPotential (Macros.hpp:486-533)
struct Potential {
  double mass = 0, factor = 0, rcut = 0;
  Spline rho, embed, pair, u, w;
};
Potential gMgMg, gHH, gMgH;
double gMass[32];

bool read_spline(FILE *f, Spline &s) {
  if (fscanf(f, "%d %lf", &s.n, &s.dx) != 2) return false;
  std::vector<double> *cols[9] = {&s.a, &s.b, &s.c, &s.d, &s.db,
                                  &s.dc, &s.dd, &s.ddc, &s.ddd};
  for (auto *c : cols) c->assign(s.n, 0.0);
  for (int i = 0; i < s.n; ++i)
    for (auto *c : cols)
      if (fscanf(f, "%lf", &(*c)[i]) != 1) return false;
  return true;
}

// init_adp_MgHx (MgHx-ADP.cpp:366-501): element files hold
// "mass factor rcut", rho and embedding splines, then pair/u/w splines; the
// alloy file holds "rcut" and the pair/u/w splines only.
bool load_potential(const std::string &path, Potential &p, bool alloy) {
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return false;
  bool ok = true;
  if (!alloy) {
    ok = fscanf(f, "%lf %lf %lf", &p.mass, &p.factor, &p.rcut) == 3;
    ok = ok && read_spline(f, p.rho) && read_spline(f, p.embed);
  } else {
    ok = fscanf(f, "%lf", &p.rcut) == 1;
  }
  ok = ok && read_spline(f, p.pair) && read_spline(f, p.u) && read_spline(f, p.w);
  fclose(f);
  return ok;
}

const Spline *table_by_id(int id) {
  switch (id) {
  case 0: return &gMgMg.rho;
  case 1: return &gHH.rho;
  case 2: return &gMgMg.embed;
  case 3: return &gHH.embed;
  case 4: return &gMgMg.pair;
  case 5: return &gHH.pair;
  case 6: return &gMgH.pair;
  case 7: return &gMgMg.u;
  case 8: return &gHH.u;
  case 9: return &gMgH.u;
  case 10: return &gMgMg.w;
  case 11: return &gHH.w;
  case 12: return &gMgH.w;
  }
  return nullptr;
}

// Table choice: rho by the species of j (MgHx-ADP.cpp:535-540); pair, u, w:
// Mg-Mg, H-H, else the Mg-H table (MgHx-ADP.cpp:881-888, 1247-1263).
const Potential &pot_of(int si, int sj) {
  if (si == kMg && sj == kMg) return gMgMg;
  if (si == kH && sj == kH) return gHH;
  return gMgH;
}
const Spline &rho_of(int sj) { return sj == kMg ? gMgMg.rho : gHH.rho; }
const Spline &embed_of(int si) { return si == kMg ? gMgMg.embed : gHH.embed; }

inline double sq(double a) { return a == 0.0 ? 0.0 : a * a; }  // DSQR

// ---------------------------------------------------------------------------
// ADP per-term functions.  Argument layout as potential_function
// (Macros.hpp:252-278): n[] occupancies, q[] 3 coordinates per slot.

// rho_ij (MgHx-ADP.cpp:526-553), d_rho_ij_dq (557-601), d_rho_ij_dn (815-844)
double rho_F(const double *n, const double *q, const int *spc) {
  double r2 = 0, r[3];
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sq(r[a]);
  }
  return n[1] * spline_val(rho_of(spc[1]), std::sqrt(r2));
}
void rho_dq(int dir, double *out, const double *n, const double *q,
            const int *spc) {
  double r2 = 0, r[3];
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sq(r[a]);
  }
  double nr = std::sqrt(r2), inv = 1.0 / nr;
  double g = n[1] * spline_d1(rho_of(spc[1]), nr);
  for (int a = 0; a < 3; ++a) out[a] = 0.0;
  if (dir == 0)
    for (int a = 0; a < 3; ++a) out[a] = g * inv * r[a];
  if (dir == 1)
    for (int a = 0; a < 3; ++a) out[a] = -g * inv * r[a];
}
double rho_dn(int dir, const double *n, const double *q, const int *spc) {
  (void)n;
  double r2 = 0, r[3];
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sq(r[a]);
  }
  return dir == 1 ? spline_val(rho_of(spc[1]), std::sqrt(r2)) : 0.0;
}

// V_pair_ij (869-900), dV_pair_ij_dq (904-949), dV_pair_ij_dn (1170-1209)
double pair_F(const double *n, const double *q, const int *spc) {
  double r2 = 0, r[3];
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sq(r[a]);
  }
  double phi = n[0] * n[1] * spline_val(pot_of(spc[0], spc[1]).pair, std::sqrt(r2));
  return 0.5 * phi;
}
void pair_dq(int dir, double *out, const double *n, const double *q,
             const int *spc) {
  double r2 = 0, r[3];
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sq(r[a]);
  }
  double nr = std::sqrt(r2), inv = 1.0 / nr;
  double g = n[0] * n[1] * spline_d1(pot_of(spc[0], spc[1]).pair, nr);
  for (int a = 0; a < 3; ++a) out[a] = 0.0;
  if (dir == 0)
    for (int a = 0; a < 3; ++a) out[a] = 0.5 * g * inv * r[a];
  if (dir == 1)
    for (int a = 0; a < 3; ++a) out[a] = -0.5 * g * inv * r[a];
}
double pair_dn(int dir, const double *n, const double *q, const int *spc) {
  double r2 = 0, r[3];
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sq(r[a]);
  }
  double phi = spline_val(pot_of(spc[0], spc[1]).pair, std::sqrt(r2));
  if (dir == 0) return 0.5 * (n[1] * phi);
  if (dir == 1) return 0.5 * (n[0] * phi);
  return 0.0;
}

// Shared geometry of the triplet terms (i = slot 0, j1 = 1, j2 = 2).
struct Tri {
  double r1[3], r2[3], r1sq = 0, r2sq = 0, dot = 0, n1, n2;
};
Tri tri_geom(const double *q) {
  Tri t;
  for (int a = 0; a < 3; ++a) {
    t.r1[a] = q[a] - q[3 + a];
    t.r2[a] = q[a] - q[6 + a];
    t.r1sq += sq(t.r1[a]);
    t.r2sq += sq(t.r2[a]);
    t.dot += t.r1[a] * t.r2[a];
  }
  t.n1 = std::sqrt(t.r1sq);
  t.n2 = std::sqrt(t.r2sq);
  return t;
}

// V_dipole_ij1j2 (1233-1281), dV_dipole_ij1j2_dq (1285-1371), _dn (1683-1758)
double dip_F(const double *n, const double *q, const int *spc) {
  Tri t = tri_geom(q);
  double u1 = n[0] * n[1] * spline_val(pot_of(spc[0], spc[1]).u, t.n1);
  double u2 = n[0] * n[2] * spline_val(pot_of(spc[0], spc[2]).u, t.n2);
  return (1.0 / 2.0) * u1 * u2 * t.dot;
}
void dip_dq(int dir, double *out, const double *n, const double *q,
            const int *spc) {
  Tri t = tri_geom(q);
  const Spline &s1 = pot_of(spc[0], spc[1]).u, &s2 = pot_of(spc[0], spc[2]).u;
  double i1 = 1.0 / t.n1, i2 = 1.0 / t.n2;
  double u1 = n[0] * n[1] * spline_val(s1, t.n1);
  double u2 = n[0] * n[2] * spline_val(s2, t.n2);
  double du1 = n[0] * n[1] * spline_d1(s1, t.n1);
  double du2 = n[0] * n[2] * spline_d1(s2, t.n2);
  for (int a = 0; a < 3; ++a) out[a] = 0.0;
  for (int a = 0; a < 3; ++a) {
    if (dir == 0)
      out[a] = 0.5 * (du1 * u2 * t.dot * i1 * t.r1[a] +
                      u1 * du2 * t.dot * i2 * t.r2[a] +
                      u1 * u2 * (t.r1[a] + t.r2[a]));
    if (dir == 1)
      out[a] = -0.5 * (du1 * u2 * t.dot * i1 * t.r1[a] + u1 * u2 * t.r2[a]);
    if (dir == 2)
      out[a] = -0.5 * (u1 * du2 * t.dot * i2 * t.r2[a] + u1 * u2 * t.r1[a]);
  }
}
double dip_dn(int dir, const double *n, const double *q, const int *spc) {
  Tri t = tri_geom(q);
  double s1 = spline_val(pot_of(spc[0], spc[1]).u, t.n1);
  double s2 = spline_val(pot_of(spc[0], spc[2]).u, t.n2);
  if (dir == 0) {
    double u1 = n[0] * n[1] * s1, u2 = n[0] * n[2] * s2;
    double d1 = n[1] * s1, d2 = n[2] * s2;
    return (1.0 / 2.0) * d1 * u2 * t.dot + (1.0 / 2.0) * u1 * d2 * t.dot;
  }
  if (dir == 1) return (1.0 / 2.0) * (n[0] * s1) * (n[0] * n[2] * s2) * t.dot;
  if (dir == 2) return (1.0 / 2.0) * (n[0] * n[1] * s1) * (n[0] * s2) * t.dot;
  return 0.0;
}

// V_quadrupole_ij1j2 (1781-1831), _dq (1835-1935), _dn (2352-2434)
double quad_F(const double *n, const double *q, const int *spc) {
  Tri t = tri_geom(q);
  double w1 = n[0] * n[1] * spline_val(pot_of(spc[0], spc[1]).w, t.n1);
  double w2 = n[0] * n[2] * spline_val(pot_of(spc[0], spc[2]).w, t.n2);
  return (1.0 / 2.0) * w1 * w2 * sq(t.dot) -
         (1.0 / 6.0) * w1 * w2 * t.r1sq * t.r2sq;
}
void quad_dq(int dir, double *out, const double *n, const double *q,
             const int *spc) {
  Tri t = tri_geom(q);
  const Spline &s1 = pot_of(spc[0], spc[1]).w, &s2 = pot_of(spc[0], spc[2]).w;
  double i1 = 1.0 / t.n1, i2 = 1.0 / t.n2, dd = sq(t.dot);
  double w1 = n[0] * n[1] * spline_val(s1, t.n1);
  double w2 = n[0] * n[2] * spline_val(s2, t.n2);
  double dw1 = n[0] * n[1] * spline_d1(s1, t.n1);
  double dw2 = n[0] * n[2] * spline_d1(s2, t.n2);
  for (int a = 0; a < 3; ++a) out[a] = 0.0;
  for (int a = 0; a < 3; ++a) {
    if (dir == 0)
      out[a] = (1.0 / 2.0) * (dw1 * w2 * dd * i1 * t.r1[a] +
                              w1 * dw2 * dd * i2 * t.r2[a] +
                              w1 * w2 * 2 * t.dot * (t.r1[a] + t.r2[a])) -
               (1.0 / 6.0) * (dw1 * w2 * t.n1 * t.r2sq * t.r1[a] +
                              w1 * dw2 * t.r1sq * t.n2 * t.r2[a] +
                              w1 * w2 * 2 * t.r2sq * t.r1[a] +
                              w1 * w2 * 2 * t.r1sq * t.r2[a]);
    if (dir == 1)
      out[a] = -0.5 * (dw1 * w2 * dd * i1 * t.r1[a] +
                       w1 * w2 * 2 * t.dot * t.r2[a]) +
               (1.0 / 6.0) * (dw1 * w2 * t.n1 * t.r2sq * t.r1[a] +
                              w1 * w2 * 2 * t.r2sq * t.r1[a]);
    if (dir == 2)
      out[a] = -0.5 * (w1 * dw2 * dd * i2 * t.r2[a] +
                       w1 * w2 * 2 * t.dot * t.r1[a]) +
               (1.0 / 6.0) * (w1 * dw2 * t.r1sq * t.n2 * t.r2[a] +
                              w1 * w2 * 2 * t.r1sq * t.r2[a]);
  }
}
double quad_dn(int dir, const double *n, const double *q, const int *spc) {
  Tri t = tri_geom(q);
  double s1 = spline_val(pot_of(spc[0], spc[1]).w, t.n1);
  double s2 = spline_val(pot_of(spc[0], spc[2]).w, t.n2);
  if (dir == 0) {
    double w1 = n[0] * n[1] * s1, w2 = n[0] * n[2] * s2;
    double d1 = n[1] * s1, d2 = n[2] * s2, dd = sq(t.dot);
    return (1.0 / 2.0) * d1 * w2 * dd + (1.0 / 2.0) * w1 * d2 * dd -
           (1.0 / 6.0) * d1 * w2 * t.r1sq * t.r2sq -
           (1.0 / 6.0) * w1 * d2 * t.r1sq * t.r2sq;
  }
  if (dir == 1) {
    double d1 = n[0] * s1, w2 = n[0] * n[2] * s2;
    return (1.0 / 2.0) * d1 * w2 * sq(t.dot) -
           (1.0 / 6.0) * d1 * w2 * t.r1sq * t.r2sq;
  }
  if (dir == 2) {
    double w1 = n[0] * n[1] * s1, d2 = n[0] * s2;
    return (1.0 / 2.0) * w1 * d2 * sq(t.dot) -
           (1.0 / 6.0) * w1 * d2 * t.r1sq * t.r2sq;
  }
  return 0.0;
}

struct Term {
  double (*F)(const double *, const double *, const int *);
  void (*dq)(int, double *, const double *, const double *, const int *);
  double (*dn)(int, const double *, const double *, const int *);
  int id;  // 0 rho, 1 pair, 2 dipole, 3 quadrupole
};
const Term kRho = {rho_F, rho_dq, rho_dn, 0};
const Term kPair = {pair_F, pair_dq, pair_dn, 1};
const Term kDip = {dip_F, dip_dq, dip_dn, 2};
const Term kQuad = {quad_F, quad_dq, quad_dn, 3};

// The integration rule behind the reference's compile switch
// (MgHx-mf-V-bulk.cpp:715-724): 0 the degree-3 Gauss-Hermite rule
// (GH3TH_INTEGRAL, the shipped build); 1 the multipole rule
// (MULTIPOLE_INTEGRAL) as the reference's build flags compile it, whose
// `#ifdef NUMERICAL_DERIVATIVES` (Quadrature-Multipole.cpp:134, 185) holds
// under CMakeLists.txt:185's -DNUMERICAL_DERIVATIVES=0 and selects the
// finite-difference Hessians; 2 the multipole rule with the analytic
// Hessians (NUMERICAL_DERIVATIVES undefined).  The occupancy derivative
// always uses the degree-3 rule (meanfield_integral_gh_3th_dxi, 2160-2257).
int gRule = 0;

// ---------------------------------------------------------------------------
// Gaussian measure (Quadrature-Measure.cpp:30-109): reduce the dof table so
// coincident sites form one group, then one integration row per axis of each
// group.  board[row][3*site+axis] = 1 where that row moves that site.
struct Measure {
  int ns = 0, D = 0;
  int board[9][9];
  int dof[9];
  const double *mean, *sigma, *x;
  const int *spc;
};

Measure make_measure(const double *mean, const double *sigma, const double *x,
                     const int *spc, const int *dof, int ns) {
  Measure m;
  m.ns = ns;
  m.mean = mean;
  m.sigma = sigma;
  m.x = x;
  m.spc = spc;
  int aux[3][3];
  for (int k = 0; k < ns * ns; ++k) m.dof[k] = dof[k];
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) aux[i][j] = dof[i * ns + j];
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j)
      if (j != i)
        for (int k = 0; k < ns; ++k)
          if (aux[j][k] == aux[i][k]) aux[j][k] = 0;
  memset(m.board, 0, sizeof(m.board));
  int row = 0;
  for (int i = 0; i < ns; ++i) {
    int cnt = 0;
    for (int j = 0; j < ns; ++j) cnt += aux[i][j];
    if (cnt <= 0) continue;
    for (int j = 0; j < ns; ++j)
      if (aux[i][j])
        for (int k = 0; k < 3; ++k) m.board[row * 3 + k][j * 3 + k] = 1;
    ++row;
  }
  m.D = row * 3;
  return m;
}

// Degree-3 rule (Quadrature-Hermitian-3th.cpp:36-110): 2D points
// q = mean +/- sqrt(2) sigma zeta board_l, zeta = sqrt(D)/sqrt(2), weight 1/(2D).
void point(const Measure &m, int l, double sgn, double *ql) {
  double zeta = std::sqrt((double)m.D) / kSqrt2;
  for (int s = 0; s < m.ns; ++s)
    for (int a = 0; a < 3; ++a) {
      double off = kSqrt2 * m.sigma[s] * zeta * m.board[l][s * 3 + a];
      ql[s * 3 + a] = sgn > 0 ? m.mean[s * 3 + a] + off : m.mean[s * 3 + a] - off;
    }
}

double integ_mp(const Term &f, const Measure &m);
void integ_mp_dmq(int dir, const Term &f, const Measure &m, double *out);
double integ_mp_dsq(int dir, const Term &f, const Measure &m);

double integ(const Term &f, const Measure &m) {
  if (gRule != 0) return integ_mp(f, m);
  double W = 1.0 / (2.0 * m.D), acc = 0.0, ql[9];
  for (double sgn : {1.0, -1.0})
    for (int l = 0; l < m.D; ++l) {
      point(m, l, sgn, ql);
      acc += f.F(m.x, ql, m.spc) * W;
    }
  return acc;
}

// meanfield_integral_gh_3th_dmq (212-296)
void integ_dmq(int dir, const Term &f, const Measure &m, double *out) {
  if (gRule != 0) return integ_mp_dmq(dir, f, m, out);
  double W = 1.0 / (2.0 * m.D), ql[9], g[3];
  for (int a = 0; a < 3; ++a) out[a] = 0.0;
  for (double sgn : {1.0, -1.0})
    for (int l = 0; l < m.D; ++l) {
      point(m, l, sgn, ql);
      f.dq(dir, g, m.x, ql, m.spc);
      for (int a = 0; a < 3; ++a) out[a] += g[a] * W;
    }
}

// meanfield_integral_gh3th_dsq (114-208)
double integ_dsq(int dir, const Term &f, const Measure &m) {
  if (gRule != 0) return integ_mp_dsq(dir, f, m);
  double W = 1.0 / (2.0 * m.D), ql[9], g[3], acc = 0.0;
  double zeta = std::sqrt((double)m.D) / kSqrt2;
  for (double sgn : {1.0, -1.0})
    for (int l = 0; l < m.D; ++l) {
      point(m, l, sgn, ql);
      double dqds[3];
      for (int a = 0; a < 3; ++a)
        dqds[a] = sgn * kSqrt2 * zeta * m.board[l][dir * 3 + a];
      f.dq(dir, g, m.x, ql, m.spc);
      for (int a = 0; a < 3; ++a) acc += g[a] * dqds[a] * W;
    }
  return acc;
}

// meanfield_integral_gh_3th_dxi (300-378)
double integ_dxi(int dir, const Term &f, const Measure &m) {
  double W = 1.0 / (2.0 * m.D), ql[9], acc = 0.0;
  for (double sgn : {1.0, -1.0})
    for (int l = 0; l < m.D; ++l) {
      point(m, l, sgn, ql);
      acc += f.dn(dir, m.x, ql, m.spc) * W;
    }
  return acc;
}

// ---------------------------------------------------------------------------
// Per-site drivers.
struct View {
  const double *q, *sigma, *x, *rho;
  const int *spc, *offs, *idx;
};

struct PairCtx {
  double mean[6], sig[2], xx[2];
  int sp[2];
  Measure m;
};
void pair_ctx(const View &v, int i, int j, PairCtx &c) {
  for (int a = 0; a < 3; ++a) {
    c.mean[a] = v.q[3 * i + a];
    c.mean[3 + a] = v.q[3 * j + a];
  }
  c.sig[0] = v.sigma[i];
  c.sig[1] = v.sigma[j];
  c.xx[0] = v.x[i];
  c.xx[1] = v.x[j];
  c.sp[0] = v.spc[i];
  c.sp[1] = v.spc[j];
  static const int dof[4] = {1, 0, 0, 1};
  c.m = make_measure(c.mean, c.sig, c.xx, c.sp, dof, 2);
}

struct TriCtx {
  double mean[9], sig[3], xx[3];
  int sp[3];
  Measure m;
};
void tri_ctx(const View &v, int i, int j1, int j2, TriCtx &c) {
  int s[3] = {i, j1, j2};
  for (int k = 0; k < 3; ++k) {
    for (int a = 0; a < 3; ++a) c.mean[3 * k + a] = v.q[3 * s[k] + a];
    c.sig[k] = v.sigma[s[k]];
    c.xx[k] = v.x[s[k]];
    c.sp[k] = v.spc[s[k]];
  }
  int dof[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (j1 == j2) {  // MgHx-mf-V-bulk.cpp:892-895
    dof[5] = 1;
    dof[7] = 1;
  }
  c.m = make_measure(c.mean, c.sig, c.xx, c.sp, dof, 3);
}

// evaluate_mf_rho_i_adp_MgHx (MgHx-mf-V-bulk.cpp:708-787)
double mf_rho_i(const View &v, int i) {
  if (v.spc[i] == kH && v.x[i] < kMinOcc) return 0.0;
  double acc = 0.0;
  for (int k = v.offs[i]; k < v.offs[i + 1]; ++k) {
    int j = v.idx[k];
    if (v.spc[j] == kH && v.x[j] < kMinOcc) continue;
    PairCtx c;
    pair_ctx(v, i, j, c);
    acc += integ(kRho, c.m);
  }
  return acc;
}

// Mean-field <V>_0 of site i (evaluate_V0_i_adp_MgHx, 791-953); `skip_any`
// selects the any-species site test of evaluate_S0_i_adp_MgHx (1004).
double V0_i(const View &v, int i) {
  double xi = v.x[i];
  double pair = 0, dip = 0, quad = 0;
  int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    int j1 = v.idx[k1];
    if (v.spc[j1] == kH && v.x[j1] < kMinOcc) continue;
    PairCtx c;
    pair_ctx(v, i, j1, c);
    pair += integ(kPair, c.m);
    for (int k2 = k1; k2 < nb1; ++k2) {
      int j2 = v.idx[k2];
      if (v.x[j2] < kMinOcc) continue;
      TriCtx t;
      tri_ctx(v, i, j1, j2, t);
      double f = (k2 == k1) ? 1.0 : 2.0;
      dip += f * integ(kDip, t.m);
      quad += f * integ(kQuad, t.m);
    }
  }
  double emb = xi * spline_val(embed_of(v.spc[i]), v.rho[i]);
  return emb + pair + dip + quad;
}

// evaluate_DV0_i_Dq_u_MgHx (1823-2098): (dV0_i/dmean_q_u, dV0_i/dsigma_u).
void DV0_dq(const View &v, int u, int i, double *out4) {
  for (int c = 0; c < 4; ++c) out4[c] = 0.0;
  if (v.x[u] < kMinOcc) return;
  if (v.x[i] < kMinOcc) return;
  double drho_q[3] = {0, 0, 0}, pair_q[3] = {0, 0, 0};
  double dip_q[3] = {0, 0, 0}, quad_q[3] = {0, 0, 0};
  double drho_s = 0, pair_s = 0, dip_s = 0, quad_s = 0;
  int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    int j1 = v.idx[k1];
    if (v.x[j1] < kMinOcc) continue;
    PairCtx c;
    pair_ctx(v, i, j1, c);
    int sites2[2] = {i, j1};
    for (int dir = 0; dir < 2; ++dir) {
      if (sites2[dir] != u) continue;
      double g[3];
      integ_dmq(dir, kRho, c.m, g);
      for (int a = 0; a < 3; ++a) drho_q[a] += g[a];
      integ_dmq(dir, kPair, c.m, g);
      for (int a = 0; a < 3; ++a) pair_q[a] += g[a];
      drho_s += integ_dsq(dir, kRho, c.m);
      pair_s += integ_dsq(dir, kPair, c.m);
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      int j2 = v.idx[k2];
      if (v.x[j2] <= kMinOcc) continue;
      int sites3[3] = {i, j1, j2};
      if (sites3[0] != u && sites3[1] != u && sites3[2] != u) continue;
      TriCtx t;
      tri_ctx(v, i, j1, j2, t);
      double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        if (sites3[dir] != u) continue;
        double g[3];
        integ_dmq(dir, kDip, t.m, g);
        for (int a = 0; a < 3; ++a) dip_q[a] += f * g[a];
        integ_dmq(dir, kQuad, t.m, g);
        for (int a = 0; a < 3; ++a) quad_q[a] += f * g[a];
        dip_s += f * integ_dsq(dir, kDip, t.m);
        quad_s += f * integ_dsq(dir, kQuad, t.m);
      }
    }
  }
  double dF = spline_d1(embed_of(v.spc[i]), v.rho[i]);
  for (int a = 0; a < 3; ++a)
    out4[a] = v.x[i] * dF * drho_q[a] + pair_q[a] + dip_q[a] + quad_q[a];
  out4[3] = v.x[i] * dF * drho_s + pair_s + dip_s + quad_s;
}

// evaluate_DV0_i_Dxi_u_adp_MgHx (2102-2325)
double DV0_dx(const View &v, int u, int i) {
  if (v.x[u] < kMinOcc) return 0.0;
  if (v.x[i] < kMinOcc) return 0.0;
  double drho = 0, pair = 0, dip = 0, quad = 0;
  int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    int j1 = v.idx[k1];
    if (v.x[j1] < kMinOcc) continue;
    PairCtx c;
    pair_ctx(v, i, j1, c);
    int sites2[2] = {i, j1};
    for (int dir = 0; dir < 2; ++dir) {
      if (sites2[dir] != u) continue;
      drho += integ_dxi(dir, kRho, c.m);
      pair += integ_dxi(dir, kPair, c.m);
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      int j2 = v.idx[k2];
      if (v.x[j2] < kMinOcc) continue;
      int sites3[3] = {i, j1, j2};
      if (sites3[0] != u && sites3[1] != u && sites3[2] != u) continue;
      TriCtx t;
      tri_ctx(v, i, j1, j2, t);
      double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        if (sites3[dir] != u) continue;
        dip += f * integ_dxi(dir, kDip, t.m);
        quad += f * integ_dxi(dir, kQuad, t.m);
      }
    }
  }
  double emb = 0.0;
  int si = v.spc[i];
  if (si == kH && i == u) emb = spline_val(gHH.embed, v.rho[i]);
  if (si == kH && i != u) emb = v.x[i] * spline_d1(gHH.embed, v.rho[i]) * drho;
  if (si == kMg) emb = spline_d1(gMgMg.embed, v.rho[i]) * drho;  // no x_i (2312-2315)
  return emb + pair + dip + quad;
}

// evaluate_DV0_i_dF_bulk_MgHx (MgHx-mf-V-bulk.cpp:2329-2552): sum over the
// sites a of every term of V0_i of d<term>/dmean_q_a (x) q0_a (sigma held),
// 3x3 row-major.
void DV0_dF(const View &v, const double *q0, int i, double *out9) {
  for (int c = 0; c < 9; ++c) out9[c] = 0.0;
  if (v.x[i] < kMinOcc) return;  // 2371-2373
  double drho[9] = {0}, pair[9] = {0}, dip[9] = {0}, quad[9] = {0};
  const int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    const int j1 = v.idx[k1];
    if (v.spc[j1] == kH && v.x[j1] < kMinOcc) continue;  // 2408-2410
    PairCtx c;
    pair_ctx(v, i, j1, c);
    int sites2[2] = {i, j1};
    for (int dir = 0; dir < 2; ++dir) {
      const double *r0 = q0 + 3 * sites2[dir];
      double g[3];
      integ_dmq(dir, kRho, c.m, g);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) drho[3 * a + b] += g[a] * r0[b];
      integ_dmq(dir, kPair, c.m, g);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) pair[3 * a + b] += g[a] * r0[b];
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      const int j2 = v.idx[k2];
      if (v.spc[j2] == kH && v.x[j2] < kMinOcc) continue;  // 2465-2467
      TriCtx t;
      tri_ctx(v, i, j1, j2, t);
      int sites3[3] = {i, j1, j2};
      const double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        const double *r0 = q0 + 3 * sites3[dir];
        double g[3];
        integ_dmq(dir, kDip, t.m, g);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) dip[3 * a + b] += f * g[a] * r0[b];
        integ_dmq(dir, kQuad, t.m, g);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) quad[3 * a + b] += f * g[a] * r0[b];
      }
    }
  }
  const double dF = spline_d1(embed_of(v.spc[i]), v.rho[i]);  // 2536-2543
  for (int c = 0; c < 9; ++c) out9[c] = v.x[i] * dF * drho[c] + pair[c] + dip[c] + quad[c];
}

// ---------------------------------------------------------------------------
// Non-mean-field forms: the ADP terms at the mean positions (sigma -> 0).

// evaluate_DV_i_Dq_u_adp_MgHx (MgHx-mf-V-bulk.cpp:147-330): dV_i/dq_u.  The
// reference tests u's membership per term after building it; the test is
// made first here (the value is the same).
void DV_dq(const View &v, int u, int i, double *out3) {
  for (int a = 0; a < 3; ++a) out3[a] = 0.0;
  if (v.spc[u] == kH && v.x[u] < kMinOcc) return;  // 161-165
  if (v.spc[i] == kH && v.x[i] < kMinOcc) return;  // 185-188
  double drho[3] = {0, 0, 0}, pair[3] = {0, 0, 0}, dip[3] = {0, 0, 0}, quad[3] = {0, 0, 0};
  const int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    const int j1 = v.idx[k1];
    if (v.spc[j1] == kH && v.x[j1] < kMinOcc) continue;  // 200-202
    double qq[6], nn[2] = {v.x[i], v.x[j1]};
    int sp[2] = {v.spc[i], v.spc[j1]}, sites2[2] = {i, j1};
    for (int a = 0; a < 3; ++a) {
      qq[a] = v.q[3 * i + a];
      qq[3 + a] = v.q[3 * j1 + a];
    }
    for (int dir = 0; dir < 2; ++dir) {
      if (sites2[dir] != u) continue;
      double g[3];
      rho_dq(dir, g, nn, qq, sp);
      for (int a = 0; a < 3; ++a) drho[a] += g[a];
      pair_dq(dir, g, nn, qq, sp);
      for (int a = 0; a < 3; ++a) pair[a] += g[a];
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      const int j2 = v.idx[k2];
      if (v.spc[j2] == kH && v.x[j2] < kMinOcc) continue;  // 252-254
      int sites3[3] = {i, j1, j2};
      if (sites3[0] != u && sites3[1] != u && sites3[2] != u) continue;
      double q3[9], n3[3] = {v.x[i], v.x[j1], v.x[j2]};
      int sp3[3] = {v.spc[i], v.spc[j1], v.spc[j2]};
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) q3[3 * k + a] = v.q[3 * sites3[k] + a];
      const double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        if (sites3[dir] != u) continue;
        double g[3];
        dip_dq(dir, g, n3, q3, sp3);
        for (int a = 0; a < 3; ++a) dip[a] += f * g[a];
        quad_dq(dir, g, n3, q3, sp3);
        for (int a = 0; a < 3; ++a) quad[a] += f * g[a];
      }
    }
  }
  const double dF = spline_d1(embed_of(v.spc[i]), v.rho[i]);  // 308-315
  for (int a = 0; a < 3; ++a) out3[a] = v.x[i] * dF * drho[a] + pair[a] + dip[a] + quad[a];
}

// ---- second derivatives of the point terms, restated from the terms'
// definitions (the reference's d2F_dq2 slots, MgHx-ADP.cpp:664-735,
// 1030-1090, 1380-1600, 2040-2300).  Only the diagonal blocks d2/dq_a^2 of
// one slot a are needed; with r = q_0 - q_k every block is a second
// derivative in r_k (the sign of dr/dq cancels).

// H += c (f'' rr^T/s^2 + f' (I - rr^T/s^2)/s): the Hessian of c f(|r|).
void radial_hess(const double *r, double s, double d1, double d2, double c, double *H) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double rr = r[a] * r[b] / (s * s);
      H[3 * a + b] += c * (d2 * rr + d1 * ((a == b ? 1.0 : 0.0) - rr) / s);
    }
}

// sum_al m_al d2 A_al / dr dr with A = c u(|r|) r:
//   c [u' (m r^T + r m^T)/s + (m.r)(u'' rr^T/s^2 + u' (I - rr^T/s^2)/s)]
void vec_hess(const double *m, const double *r, double s, double u1, double u2, double c,
              double *H) {
  const double mr = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double rr = r[a] * r[b] / (s * s);
      H[3 * a + b] += c * (u1 * (m[a] * r[b] + r[a] * m[b]) / s +
                           mr * (u2 * rr + u1 * ((a == b ? 1.0 : 0.0) - rr) / s));
    }
}

// sum_ab M_ab d2 B_ab / dr dr with B = c w(|r|) r r^T (M symmetric):
//   c [(r^T M r)(w'' rr^T/s^2 + w' (I - rr^T/s^2)/s)
//      + 2 w' (r (Mr)^T + (Mr) r^T)/s + 2 w M]
void ten_hess(const double *M, const double *r, double s, double w0, double w1, double w2,
              double c, double *H) {
  double Mr[3];
  for (int a = 0; a < 3; ++a) Mr[a] = M[3 * a] * r[0] + M[3 * a + 1] * r[1] + M[3 * a + 2] * r[2];
  const double rMr = r[0] * Mr[0] + r[1] * Mr[1] + r[2] * Mr[2];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double rr = r[a] * r[b] / (s * s);
      H[3 * a + b] += c * (rMr * (w2 * rr + w1 * ((a == b ? 1.0 : 0.0) - rr) / s) +
                           2.0 * w1 * (r[a] * Mr[b] + Mr[a] * r[b]) / s + 2.0 * w0 * M[3 * a + b]);
    }
}

// d2/dq_a^2 of V_dip(0, 1, 2) = 1/2 A1.A2, A_k = n0 n_k u(|r_k|) r_k: block
// a = 0 moves both r_k, blocks 1 and 2 move r_1 or r_2 alone.
void dip_d2(int a, const double *n, const double *q, const int *spc, double *H) {
  for (int c = 0; c < 9; ++c) H[c] = 0.0;
  Tri t = tri_geom(q);
  const Spline &S1 = pot_of(spc[0], spc[1]).u, &S2 = pot_of(spc[0], spc[2]).u;
  const double c1 = n[0] * n[1], c2 = n[0] * n[2];
  const double u1 = spline_val(S1, t.n1), du1 = spline_d1(S1, t.n1), dd1 = spline_d2(S1, t.n1);
  const double u2 = spline_val(S2, t.n2), du2 = spline_d1(S2, t.n2), dd2 = spline_d2(S2, t.n2);
  double A1[3], A2[3];
  for (int k = 0; k < 3; ++k) {
    A1[k] = c1 * u1 * t.r1[k];
    A2[k] = c2 * u2 * t.r2[k];
  }
  double h[9] = {0};
  if (a == 0 || a == 1) vec_hess(A2, t.r1, t.n1, du1, dd1, c1, h);
  if (a == 0 || a == 2) vec_hess(A1, t.r2, t.n2, du2, dd2, c2, h);
  if (a == 0) {  // J1^T J2 + J2^T J1, J_k = c_k (u I + u' r r^T / s)
    double J1[9], J2[9];
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) {
        J1[3 * x + y] = c1 * ((x == y ? u1 : 0.0) + du1 * t.r1[x] * t.r1[y] / t.n1);
        J2[3 * x + y] = c2 * ((x == y ? u2 : 0.0) + du2 * t.r2[x] * t.r2[y] / t.n2);
      }
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y)
        for (int z = 0; z < 3; ++z)
          h[3 * x + y] += J1[3 * z + x] * J2[3 * z + y] + J2[3 * z + x] * J1[3 * z + y];
  }
  for (int c = 0; c < 9; ++c) H[c] = 0.5 * h[c];
}

// d2/dq_a^2 of V_quad(0, 1, 2) = 1/2 B1:B2 - 1/6 t1 t2, B_k = n0 n_k w r_k r_k^T,
// t_k = tr B_k = n0 n_k w s_k^2.
void quad_d2(int a, const double *n, const double *q, const int *spc, double *H) {
  for (int c = 0; c < 9; ++c) H[c] = 0.0;
  Tri t = tri_geom(q);
  const Spline &S1 = pot_of(spc[0], spc[1]).w, &S2 = pot_of(spc[0], spc[2]).w;
  const double c1 = n[0] * n[1], c2 = n[0] * n[2];
  const double w1 = spline_val(S1, t.n1), dw1 = spline_d1(S1, t.n1), ddw1 = spline_d2(S1, t.n1);
  const double w2 = spline_val(S2, t.n2), dw2 = spline_d1(S2, t.n2), ddw2 = spline_d2(S2, t.n2);
  double B1[9], B2[9];
  for (int x = 0; x < 3; ++x)
    for (int y = 0; y < 3; ++y) {
      B1[3 * x + y] = c1 * w1 * t.r1[x] * t.r1[y];
      B2[3 * x + y] = c2 * w2 * t.r2[x] * t.r2[y];
    }
  const double t1 = c1 * w1 * t.r1sq, t2 = c2 * w2 * t.r2sq;
  // trace terms: h(s) = w s^2, h' = w' s^2 + 2 w s, h'' = w'' s^2 + 4 w' s + 2 w
  const double hp1 = dw1 * t.r1sq + 2.0 * w1 * t.n1, hpp1 = ddw1 * t.r1sq + 4.0 * dw1 * t.n1 + 2.0 * w1;
  const double hp2 = dw2 * t.r2sq + 2.0 * w2 * t.n2, hpp2 = ddw2 * t.r2sq + 4.0 * dw2 * t.n2 + 2.0 * w2;
  double h[9] = {0};
  if (a == 0 || a == 1) {
    ten_hess(B2, t.r1, t.n1, w1, dw1, ddw1, 0.5 * c1, h);
    radial_hess(t.r1, t.n1, hp1, hpp1, -t2 * c1 / 6.0, h);
  }
  if (a == 0 || a == 2) {
    ten_hess(B1, t.r2, t.n2, w2, dw2, ddw2, 0.5 * c2, h);
    radial_hess(t.r2, t.n2, hp2, hpp2, -t1 * c2 / 6.0, h);
  }
  if (a == 0) {
    // 1/2 (dB1:dB2 + dB2:dB1) - 1/6 (grad t1 grad t2^T + grad t2 grad t1^T)
    double G[9] = {0};  // sum_ab dB1_ab/dr_x dB2_ab/dr_y
    const double d12 = t.dot;
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y)
        G[3 * x + y] = c1 * c2 *
                       (dw1 * dw2 * (t.r1[x] / t.n1) * (t.r2[y] / t.n2) * d12 * d12 +
                        2.0 * dw1 * w2 * (t.r1[x] / t.n1) * t.r1[y] * d12 +
                        2.0 * w1 * dw2 * t.r2[x] * (t.r2[y] / t.n2) * d12 +
                        2.0 * w1 * w2 * ((x == y ? d12 : 0.0) + t.r2[x] * t.r1[y]));
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) {
        const double g1x = c1 * hp1 * t.r1[x] / t.n1, g1y = c1 * hp1 * t.r1[y] / t.n1;
        const double g2x = c2 * hp2 * t.r2[x] / t.n2, g2y = c2 * hp2 * t.r2[y] / t.n2;
        h[3 * x + y] += 0.5 * (G[3 * x + y] + G[3 * y + x]) - (g1x * g2y + g2x * g1y) / 6.0;
      }
  }
  for (int c = 0; c < 9; ++c) H[c] = h[c];
}

// evaluate_D2V_i_Dq2_u_MgHx (MgHx-mf-V-bulk.cpp:333-528): d2V_i/dq_u^2 as
// the reference forms it, from the diagonal blocks of the slots holding u
// (for j1 = j2 = u the two slot blocks, without their cross blocks).
void D2V_dq2(const View &v, int u, int i, double *out9) {
  for (int c = 0; c < 9; ++c) out9[c] = 0.0;
  if (v.x[u] < kMinOcc) return;  // 354-357
  if (v.x[i] < kMinOcc) return;  // 380-383
  double drho[3] = {0, 0, 0}, d2rho[9] = {0}, pair[9] = {0}, dip[9] = {0}, quad[9] = {0};
  const int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    const int j1 = v.idx[k1];
    if (v.x[j1] <= kMinOcc) continue;  // 398-400
    double qq[6], nn[2] = {v.x[i], v.x[j1]};
    int sp[2] = {v.spc[i], v.spc[j1]}, sites2[2] = {i, j1};
    for (int a = 0; a < 3; ++a) {
      qq[a] = v.q[3 * i + a];
      qq[3 + a] = v.q[3 * j1 + a];
    }
    double r[3], s2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      r[a] = qq[a] - qq[3 + a];
      s2 += sq(r[a]);
    }
    const double s = std::sqrt(s2);
    for (int dir = 0; dir < 2; ++dir) {
      if (sites2[dir] != u) continue;
      double g[3];
      rho_dq(dir, g, nn, qq, sp);
      for (int a = 0; a < 3; ++a) drho[a] += g[a];
      const Spline &R = rho_of(sp[1]), &P = pot_of(sp[0], sp[1]).pair;
      radial_hess(r, s, spline_d1(R, s), spline_d2(R, s), nn[1], d2rho);
      radial_hess(r, s, spline_d1(P, s), spline_d2(P, s), 0.5 * nn[0] * nn[1], pair);
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      const int j2 = v.idx[k2];
      if (v.x[j2] <= kMinOcc) continue;  // 452-454
      int sites3[3] = {i, j1, j2};
      if (sites3[0] != u && sites3[1] != u && sites3[2] != u) continue;
      double q3[9], n3[3] = {v.x[i], v.x[j1], v.x[j2]};
      int sp3[3] = {v.spc[i], v.spc[j1], v.spc[j2]};
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) q3[3 * k + a] = v.q[3 * sites3[k] + a];
      const double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        if (sites3[dir] != u) continue;
        double h[9];
        dip_d2(dir, n3, q3, sp3, h);
        for (int c = 0; c < 9; ++c) dip[c] += f * h[c];
        quad_d2(dir, n3, q3, sp3, h);
        for (int c = 0; c < 9; ++c) quad[c] += f * h[c];
      }
    }
  }
  const Spline &E = embed_of(v.spc[i]);
  const double dF = spline_d1(E, v.rho[i]), ddF = spline_d2(E, v.rho[i]);  // 512-519
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      out9[3 * a + b] = v.x[i] * ddF * drho[a] * drho[b] + v.x[i] * dF * d2rho[3 * a + b] +
                        pair[3 * a + b] + dip[3 * a + b] + quad[3 * a + b];
}

// Block a of the Hessian of term `term` (0 rho, 1 pair, 2 dipole, 3
// quadrupole) at one geometry.
void term_d2(int term, int a, const double *n, const double *q, const int *spc, double *H) {
  if (term >= 2) {
    if (term == 2) dip_d2(a, n, q, spc, H);
    else quad_d2(a, n, q, spc, H);
    return;
  }
  for (int c = 0; c < 9; ++c) H[c] = 0.0;
  double r[3], s2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    r[k] = q[k] - q[3 + k];
    s2 += sq(r[k]);
  }
  const double s = std::sqrt(s2);
  const Spline &S = term == 0 ? rho_of(spc[1]) : pot_of(spc[0], spc[1]).pair;
  radial_hess(r, s, spline_d1(S, s), spline_d2(S, s), term == 0 ? n[1] : 0.5 * n[0] * n[1], H);
}

// meanfield_integral_gh_3th_d2mq (Quadrature-Hermitian-3th.cpp:382-463):
// the block averaged over the rule's points.
void integ_d2(int term, int a, const Measure &m, double *out9) {
  const double W = 1.0 / (2.0 * m.D);
  double ql[9], h[9];
  for (int c = 0; c < 9; ++c) out9[c] = 0.0;
  for (double sgn : {1.0, -1.0})
    for (int l = 0; l < m.D; ++l) {
      point(m, l, sgn, ql);
      term_d2(term, a, m.x, ql, m.spc, h);
      for (int c = 0; c < 9; ++c) out9[c] += h[c] * W;
    }
}

// ---------------------------------------------------------------------------
// Multipole rule (Quadrature-Multipole.cpp:97-288).

// Trace of the j1-j2 cross block of a triplet term (directions 5 and 7 of
// dV2_dipole_ij1j2_dq2, MgHx-ADP.cpp:1435-1603, and of
// dV2_quadrupole_ij1j2_dq2, 2000-2268; both blocks have the same trace).
// With r_k = q_0 - q_k, s_k = |r_k|, d = r_1.r_2 and c_k = n_0 n_k:
//   dipole      1/2 c1 c2 (u1' u2' d^2/(s1 s2) + u1' u2 s1 + u1 u2' s2 + 3 u1 u2)
//   quadrupole  1/2 c1 c2 d (w1' w2' d^2/(s1 s2) + 2 w1' w2 s1 + 2 w1 w2' s2 + 8 w1 w2)
//               - 1/6 c1 c2 d (w1' s1 + 2 w1)(w2' s2 + 2 w2)
double tri_cross_trace(int term, const double *n, const double *q, const int *spc) {
  Tri t = tri_geom(q);
  const double c1 = n[0] * n[1], c2 = n[0] * n[2];
  const Spline &S1 = term == 2 ? pot_of(spc[0], spc[1]).u : pot_of(spc[0], spc[1]).w;
  const Spline &S2 = term == 2 ? pot_of(spc[0], spc[2]).u : pot_of(spc[0], spc[2]).w;
  const double f1 = spline_val(S1, t.n1), d1 = spline_d1(S1, t.n1);
  const double f2 = spline_val(S2, t.n2), d2 = spline_d1(S2, t.n2);
  const double d = t.dot;
  if (term == 2)
    return 0.5 * c1 * c2 * (d1 * d2 * d * d / (t.n1 * t.n2) + d1 * f2 * t.n1 + f1 * d2 * t.n2 +
                            3.0 * f1 * f2);
  return 0.5 * c1 * c2 * d *
             (d1 * d2 * d * d / (t.n1 * t.n2) + 2.0 * d1 * f2 * t.n1 + 2.0 * f1 * d2 * t.n2 +
              8.0 * f1 * f2) -
         c1 * c2 * d * (d1 * t.n1 + 2.0 * f1) * (d2 * t.n2 + 2.0 * f2) / 6.0;
}

// Diagonal entry (al, al) of the finite-difference Hessian of block
// `direction` (d2_rho_ij_dq2_FD, MgHx-ADP.cpp:736-812; d2V_pair_ij_dq2_FD,
// 1091-1167; dV2_dipole_ij1j2_dq2_FD, 1605-1680;
// dV2_quadrupole_ij1j2_dq2_FD, 2270-2349): the five-point second difference
// (step 1e-4) of f in coordinate al of slot direction / (ns + 1).  Only the
// diagonal entries are formed.  The j1-j2 cross directions 5 and 7 map to
// slot 1 for the dipole and give zero for the quadrupole (whose FD Hessian
// forms directions 0, 4 and 8 only, 2291).
double fd_hess_diag(const Term &f, int ns, int direction, int al, const Measure &m,
                    const double *q) {
  if (f.id == 3 && direction != 0 && direction != 4 && direction != 8) return 0.0;
  const double dr = 0.0001;
  const int k = direction / (1 + ns) * 3 + al;
  double qpp[9], qp[9], qm[9], qmm[9];
  for (int c = 0; c < 3 * ns; ++c) {
    const double D = c == k ? 1.0 : 0.0;
    qpp[c] = q[c] + D * dr * 2;
    qp[c] = q[c] + D * dr;
    qm[c] = q[c] - D * dr;
    qmm[c] = q[c] - D * dr * 2;
  }
  const double f0 = f.F(m.x, q, m.spc);
  const double fpp = f.F(m.x, qpp, m.spc), fp = f.F(m.x, qp, m.spc);
  const double fm = f.F(m.x, qm, m.spc), fmm = f.F(m.x, qmm, m.spc);
  return (-fpp + 16.0 * fp - 30.0 * f0 + 16.0 * fm - fmm) / (12.0 * dr * dr);
}

// Trace of block `direction` = a * ns + b of d2F/dq2 (the reference's
// d2F_dq2 convention), analytic.  The dof tables of the pair and triplet
// measures request the diagonal blocks and, for j1 = j2, the j1-j2 cross
// blocks.
double block_trace(const Term &f, int ns, int direction, const Measure &m, const double *q) {
  const int a = direction / ns, b = direction % ns;
  if (a == b) {
    double H[9];
    term_d2(f.id, a, m.x, q, m.spc, H);
    return H[0] + H[4] + H[8];
  }
  if (ns == 3 && a > 0 && b > 0) return tri_cross_trace(f.id, m.x, q, m.spc);
  return 0.0;
}

// meanfield_integral_mp (Quadrature-Multipole.cpp:97-143):
//   f(mean) + sum_{(a, b) in dof} sigma_a^2 / 2 tr d2f/dq_a dq_b.
double integ_mp(const Term &f, const Measure &m) {
  double acc = f.F(m.x, m.mean, m.spc);
  for (int a = 0; a < m.ns; ++a) {
    const double c2 = sq(m.sigma[a]) / 2.0;
    for (int b = 0; b < m.ns; ++b) {
      if (m.dof[a * m.ns + b] != 1) continue;
      if (gRule == 1)
        for (int al = 0; al < 3; ++al) acc += c2 * fd_hess_diag(f, m.ns, a * m.ns + b, al, m, m.mean);
      else
        acc += c2 * block_trace(f, m.ns, a * m.ns + b, m, m.mean);
    }
  }
  return acc;
}

// meanfield_integral_mp_dsq (147-196): sigma_dir sum_{b in dof row dir} tr
// d2f/dq_dir dq_b.
double integ_mp_dsq(int dir, const Term &f, const Measure &m) {
  double acc = 0.0;
  for (int b = 0; b < m.ns; ++b) {
    if (m.dof[dir * m.ns + b] != 1) continue;
    if (gRule == 1)
      for (int al = 0; al < 3; ++al)
        acc += m.sigma[dir] * fd_hess_diag(f, m.ns, dir * m.ns + b, al, m, m.mean);
    else
      acc += m.sigma[dir] * block_trace(f, m.ns, dir * m.ns + b, m, m.mean);
  }
  return acc;
}

// meanfield_integral_mp_dmq (200-286): grad_dir f(mean) plus, for every
// site slot s and axis al, sigma_s^2 / 2 times the five-point second
// difference (step 0.01) of grad_dir f in q_{s, al}.  Each slot moves
// alone, also when two slots hold the same site.
void integ_mp_dmq(int dir, const Term &f, const Measure &m, double *out) {
  const double dr = 0.01;
  double g0[3], gpp[3], gp[3], gm[3], gmm[3], qk[9];
  f.dq(dir, g0, m.x, m.mean, m.spc);
  for (int a = 0; a < 3; ++a) out[a] = g0[a];
  for (int k = 0; k < 3 * m.ns; ++k) qk[k] = m.mean[k];
  for (int s = 0; s < m.ns; ++s) {
    const double c2 = sq(m.sigma[s]) / 2.0;
    for (int al = 0; al < 3; ++al) {
      const int k = 3 * s + al;
      qk[k] = m.mean[k] + dr * 2;
      f.dq(dir, gpp, m.x, qk, m.spc);
      qk[k] = m.mean[k] + dr;
      f.dq(dir, gp, m.x, qk, m.spc);
      qk[k] = m.mean[k] - dr;
      f.dq(dir, gm, m.x, qk, m.spc);
      qk[k] = m.mean[k] - dr * 2;
      f.dq(dir, gmm, m.x, qk, m.spc);
      qk[k] = m.mean[k];
      for (int b = 0; b < 3; ++b)
        out[b] += c2 * ((-gpp[b] + 16.0 * gp[b] - 30.0 * g0[b] + 16.0 * gm[b] - gmm[b]) /
                        (12.0 * dr * dr));
    }
  }
}

// evaluate_D2V0_i_Dmeanq2_u_MgHx (MgHx-mf-V-bulk.cpp:1366-1600).
void D2V0_dq2(const View &v, int u, int i, double *out9) {
  for (int c = 0; c < 9; ++c) out9[c] = 0.0;
  if (v.spc[u] == kH && v.x[u] < kMinOcc) return;  // 1398-1402
  if (v.spc[i] == kH && v.x[i] < kMinOcc) return;  // 1424-1427
  double drho[3] = {0, 0, 0}, d2rho[9] = {0}, pair[9] = {0}, dip[9] = {0}, quad[9] = {0};
  const int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    const int j1 = v.idx[k1];
    if (v.spc[j1] == kH && v.x[j1] <= kMinOcc) continue;  // 1441-1443
    int sites2[2] = {i, j1};
    if (sites2[0] == u || sites2[1] == u) {
      PairCtx c;
      pair_ctx(v, i, j1, c);
      for (int dir = 0; dir < 2; ++dir) {
        if (sites2[dir] != u) continue;
        double g[3], h[9];
        integ_dmq(dir, kRho, c.m, g);
        for (int a = 0; a < 3; ++a) drho[a] += g[a];
        integ_d2(0, dir, c.m, h);
        for (int k = 0; k < 9; ++k) d2rho[k] += h[k];
        integ_d2(1, dir, c.m, h);
        for (int k = 0; k < 9; ++k) pair[k] += h[k];
      }
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      const int j2 = v.idx[k2];
      if (v.spc[j2] == kH && v.x[j2] <= kMinOcc) continue;  // 1500-1502
      int sites3[3] = {i, j1, j2};
      if (sites3[0] != u && sites3[1] != u && sites3[2] != u) continue;
      TriCtx t;
      tri_ctx(v, i, j1, j2, t);
      const double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        if (sites3[dir] != u) continue;
        double h[9];
        integ_d2(2, dir, t.m, h);
        for (int k = 0; k < 9; ++k) dip[k] += f * h[k];
        integ_d2(3, dir, t.m, h);
        for (int k = 0; k < 9; ++k) quad[k] += f * h[k];
      }
    }
  }
  const Spline &E = embed_of(v.spc[i]);
  const double dF = spline_d1(E, v.rho[i]), ddF = spline_d2(E, v.rho[i]);  // 1584-1591
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      out9[3 * a + b] = v.x[i] * ddF * drho[a] * drho[b] + v.x[i] * dF * d2rho[3 * a + b] +
                        pair[3 * a + b] + dip[3 * a + b] + quad[3 * a + b];
}

// evaluate_DV_i_dF_MgHx (MgHx-mf-V-bulk.cpp:530-704): sum over the sites a
// of every term of V_i of dV_i/dq_a (x) q0_a, 3x3 row-major (row: gradient
// component, column: reference-position component).
void DV_dF(const View &v, const double *q0, int i, double *out9) {
  for (int c = 0; c < 9; ++c) out9[c] = 0.0;
  if (v.x[i] < kMinOcc) return;  // 546-549
  double drho[9] = {0}, pair[9] = {0}, dip[9] = {0}, quad[9] = {0};
  const int nb0 = v.offs[i], nb1 = v.offs[i + 1];
  for (int k1 = nb0; k1 < nb1; ++k1) {
    const int j1 = v.idx[k1];
    if (v.spc[j1] == kH && v.x[j1] < kMinOcc) continue;  // 574-576
    double qq[6], nn[2] = {v.x[i], v.x[j1]};
    int sp[2] = {v.spc[i], v.spc[j1]}, sites2[2] = {i, j1};
    for (int a = 0; a < 3; ++a) {
      qq[a] = v.q[3 * i + a];
      qq[3 + a] = v.q[3 * j1 + a];
    }
    for (int dir = 0; dir < 2; ++dir) {
      const double *r0 = q0 + 3 * sites2[dir];
      double g[3];
      rho_dq(dir, g, nn, qq, sp);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) drho[3 * a + b] += g[a] * r0[b];
      pair_dq(dir, g, nn, qq, sp);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) pair[3 * a + b] += g[a] * r0[b];
    }
    for (int k2 = k1; k2 < nb1; ++k2) {
      const int j2 = v.idx[k2];
      if (v.spc[j2] == kH && v.x[j2] < kMinOcc) continue;  // 633-635
      int sites3[3] = {i, j1, j2};
      double q3[9], n3[3] = {v.x[i], v.x[j1], v.x[j2]};
      int sp3[3] = {v.spc[i], v.spc[j1], v.spc[j2]};
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) q3[3 * k + a] = v.q[3 * sites3[k] + a];
      const double f = (k1 == k2) ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        const double *r0 = q0 + 3 * sites3[dir];
        double g[3];
        dip_dq(dir, g, n3, q3, sp3);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) dip[3 * a + b] += f * g[a] * r0[b];
        quad_dq(dir, g, n3, q3, sp3);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) quad[3 * a + b] += f * g[a] * r0[b];
      }
    }
  }
  const double dF = spline_d1(embed_of(v.spc[i]), v.rho[i]);  // 688-695
  for (int c = 0; c < 9; ++c) out9[c] = v.x[i] * dF * drho[c] + pair[c] + dip[c] + quad[c];
}

// evaluate_S0_i_adp_MgHx (957-1142)
double S0_i(const View &v, int i, double beta, double gamma) {
  double xi = v.x[i];
  if (xi < kMinOcc) return 0.0;
  double V0 = V0_i(v, i);
  double m = kUma * xi * gMass[v.spc[i] < 32 ? v.spc[i] : 0];
  double H0 = 1.0 / (2.0 * beta) + V0;
  double logZ = 3.0 * std::log((v.sigma[i] * std::sqrt(m / beta)) / kHbar);
  if (xi < 1.0) logZ += std::log(1.0 / (1.0 - xi));
  double gx = 0.0;
  if (v.spc[i] == kH) gx = gamma * (xi > 0.9999 ? 0.9999 : xi);
  return -logZ + beta * H0 - gx;
}

// Parallel loop over independent sites (std::thread; BTAM_ORACLE_THREADS).
void par_for(int n, const std::function<void(int)> &fn) {
  const char *e = getenv("BTAM_ORACLE_THREADS");
  int t = e ? atoi(e) : (int)std::thread::hardware_concurrency();
  if (t < 1) t = 1;
  if (t > n) t = n;
  if (t <= 1) {
    for (int k = 0; k < n; ++k) fn(k);
    return;
  }
  std::vector<std::thread> th;
  for (int w = 0; w < t; ++w)
    th.emplace_back([&, w]() {
      for (int k = w; k < n; k += t) fn(k);
    });
  for (auto &x : th) x.join();
}

}  // namespace

// ===========================================================================
extern "C" {

void orc_set_rule(int rule) { gRule = (rule == 1 || rule == 2) ? rule : 0; }

int orc_load_tables(const char *dir) {
  std::string d(dir);
  if (!load_potential(d + "/adpmg.dat", gMgMg, false)) return 1;
  if (!load_potential(d + "/adph.dat", gHH, false)) return 1;
  if (!load_potential(d + "/adpmgh.dat", gMgH, true)) return 1;
  for (double &m : gMass) m = 0.0;
  gMass[kMg] = gMgMg.mass;  // element_mass[] (MgHx-ADP.cpp:436)
  gMass[kH] = gHH.mass;
  return 0;
}

double orc_spline(int table, double r, int deriv) {
  const Spline *s = table_by_id(table);
  if (!s || s->n == 0) return 0.0;
  if (deriv == 0) return spline_val(*s, r);
  if (deriv == 1) return spline_d1(*s, r);
  return spline_d2(*s, r);
}

int orc_table_info(int table, double *dx) {
  const Spline *s = table_by_id(table);
  if (!s) return 0;
  *dx = s->dx;
  return s->n;
}

double orc_mass(int species) { return (species >= 0 && species < 32) ? gMass[species] : 0.0; }

// Periodic images.  Orthogonal cells follow the slab test of
// DMSwarmCreateGhostAtoms (Ghosts.cpp:123-648, In_Out_Cell 913-941): for
// direction d (x fastest, n0..n26 without n13) the site must satisfy
// lo <= q < lo + rc (d = -1), hi - rc <= q < hi (d = +1), lo <= q < hi (d = 0)
// on each axis, and the copy is shifted by -d times the box edge so that it
// lies beyond the opposite face.  (The reference's own shift search,
// Ghosts.cpp:768-794, tries the zero shift first and so leaves single-rank
// copies unshifted; this is the shift it intends.)  Triclinic cells (no
// reference counterpart: the reference supports orthogonal boxes only) keep
// every image q - sum_b d_b a_b whose fractional coordinates lie in
// [-w_a, 1 + w_a), w_a = rc / (spacing of faces a); directions in the same
// order.
int orc_ghosts(int n, const double *q, const double *origin, const double *cell,
               const int *periodic, double rc, int max_ghosts, double *q_ghost,
               int *owner, int *image, int *n_ghost) {
  bool ortho = cell[1] == 0 && cell[2] == 0 && cell[3] == 0 && cell[5] == 0 &&
               cell[6] == 0 && cell[7] == 0;
  // Reciprocal rows: frac = (q - o) . b_a, with b = inverse(cell^T) rows.
  double A[3][3], B[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = cell[3 * r + c];
  double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
               A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
               A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (det == 0.0) return kErrBoxTooSmall;
  // b_a = (a_b x a_c) / det
  for (int a = 0; a < 3; ++a) {
    const double *p = A[(a + 1) % 3], *s = A[(a + 2) % 3];
    B[a][0] = (p[1] * s[2] - p[2] * s[1]) / det;
    B[a][1] = (p[2] * s[0] - p[0] * s[2]) / det;
    B[a][2] = (p[0] * s[1] - p[1] * s[0]) / det;
  }
  double w[3], lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    double bn = std::sqrt(B[a][0] * B[a][0] + B[a][1] * B[a][1] + B[a][2] * B[a][2]);
    double height = 1.0 / bn;
    if (periodic[a] && height < 2.0 * rc) return kErrBoxTooSmall;
    w[a] = rc * bn;
    lo[a] = origin[a];
    hi[a] = origin[a] + A[a][a];
  }
  int ng = 0;
  for (int i = 0; i < n; ++i) {
    const double *qi = q + 3 * i;
    for (int dir = 0; dir < 27; ++dir) {
      if (dir == 13) continue;
      int d[3] = {dir % 3 - 1, (dir / 3) % 3 - 1, dir / 9 - 1};
      bool in = true;
      for (int a = 0; a < 3; ++a)
        if (d[a] != 0 && !periodic[a]) in = false;
      if (!in) continue;
      double p[3];
      for (int a = 0; a < 3; ++a) {
        double s = qi[a];
        for (int b = 0; b < 3; ++b)
          if (d[b] != 0) s = s + (double)(-d[b]) * A[b][a];
        p[a] = s;
      }
      if (ortho) {
        // slab test on the original position (Ghosts.cpp:123-648)
        for (int a = 0; a < 3 && in; ++a) {
          if (d[a] == -1) in = qi[a] >= lo[a] && qi[a] < lo[a] + rc;
          else if (d[a] == 1) in = qi[a] >= hi[a] - rc && qi[a] < hi[a];
          else in = qi[a] >= lo[a] && qi[a] < hi[a];
        }
      } else {
        // triclinic: keep the image if it lies in the cell widened by rc
        // across every face, -w_a <= s_a < 1 + w_a
        double dq0 = p[0] - origin[0], dq1 = p[1] - origin[1], dq2 = p[2] - origin[2];
        for (int a = 0; a < 3 && in; ++a) {
          double sa = dq0 * B[a][0] + dq1 * B[a][1] + dq2 * B[a][2];
          in = sa >= -w[a] && sa < 1.0 + w[a];
        }
      }
      if (!in) continue;
      if (ng >= max_ghosts) return kErrGhostOverflow;
      for (int a = 0; a < 3; ++a) {
        q_ghost[3 * ng + a] = p[a];
        image[3 * ng + a] = -d[a];
      }
      owner[ng] = i;
      ++ng;
    }
  }
  *n_ghost = ng;
  return 0;
}

// neighbors (Neighbors.cpp:39-134), brute force, ascending j.
int orc_neighbors(int n, const double *q, double rc, int maxn, const int *query,
                  int nquery, int *offs, int *idx, int idx_cap) {
  int total = 0;
  offs[0] = 0;
  for (int k = 0; k < nquery; ++k) {
    int i = query[k], cnt = 0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double dx = q[3 * i] - q[3 * j], dy = q[3 * i + 1] - q[3 * j + 1],
             dz = q[3 * i + 2] - q[3 * j + 2];
      double r = std::sqrt((dx * dx + dy * dy) + dz * dz);
      if (r <= rc) {
        if (cnt == maxn) return kErrNeighborOverflow;
        if (total >= idx_cap) return kErrNeighborOverflow;
        idx[total++] = j;
        ++cnt;
      }
    }
    if (cnt <= 0) return kErrNoNeighbors;
    offs[k + 1] = total;
  }
  return 0;
}

int orc_quadrature(int term, int mode, int slot, int nsites, int coincident,
                   const double *q, const double *sigma, const double *x,
                   const int *spc, double *out) {
  const Term *t = term == 0 ? &kRho : term == 1 ? &kPair : term == 2 ? &kDip
                : term == 3 ? &kQuad : nullptr;
  if (!t) return 1;
  int dof2[4] = {1, 0, 0, 1};
  int dof3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (coincident) {
    dof3[5] = 1;
    dof3[7] = 1;
  }
  Measure m = make_measure(q, sigma, x, spc, nsites == 2 ? dof2 : dof3, nsites);
  if (mode == 0) out[0] = integ(*t, m);
  else if (mode == 1) integ_dmq(slot, *t, m, out);
  else if (mode == 2) out[0] = integ_dsq(slot, *t, m);
  else out[0] = integ_dxi(slot, *t, m);
  return 0;
}

void orc_mf_rho(int n, const double *q, const double *sigma, const double *x,
                const int *spc, const int *offs, const int *idx,
                const int *sites, int nsites, double *out) {
  (void)n;
  View v{q, sigma, x, nullptr, spc, offs, idx};
  par_for(nsites, [&](int k) { out[k] = mf_rho_i(v, sites[k]); });
}

void orc_V0(int n, const double *q, const double *sigma, const double *x,
            const int *spc, const double *rho, const int *offs,
            const int *idx, const int *sites, int nsites, double *out) {
  (void)n;
  View v{q, sigma, x, rho, spc, offs, idx};
  par_for(nsites, [&](int k) {
    int i = sites[k];
    // evaluate_V0_i_adp_MgHx skips empty H sites (832-834)
    out[k] = (spc[i] == kH && x[i] < kMinOcc) ? 0.0 : V0_i(v, i);
  });
}

void orc_S0(int n, const double *q, const double *sigma, const double *x,
            const int *spc, const double *rho, const double *beta,
            const double *gamma, const int *offs, const int *idx,
            const int *sites, int nsites, double *out) {
  (void)n;
  View v{q, sigma, x, rho, spc, offs, idx};
  par_for(nsites, [&](int k) {
    int i = sites[k];
    out[k] = S0_i(v, i, beta[i], gamma[i]);
  });
}

void orc_DV0_pairs(int n, const double *q, const double *sigma,
                   const double *x, const int *spc, const double *rho,
                   const int *offs, const int *idx, const int *u_list,
                   const int *i_list, int npairs, double *out4, double *out_x) {
  (void)n;
  View v{q, sigma, x, rho, spc, offs, idx};
  par_for(npairs, [&](int k) {
    if (out4) DV0_dq(v, u_list[k], i_list[k], out4 + 4 * k);
    if (out_x) out_x[k] = DV0_dx(v, u_list[k], i_list[k]);
  });
}

// evaluate_rho_i_adp_MgHx_kokkos (density.cpp:44-104)
void orc_rho_nmf(int n, const double *q, const double *x, const int *spc,
                 const int *offs, const int *idx, const int *sites, int nsites,
                 double *out) {
  (void)n;
  par_for(nsites, [&](int k) {
    int i = sites[k];
    double acc = 0.0;
    if (!(x[i] < kMinOcc)) {
      for (int p = offs[i]; p < offs[i + 1]; ++p) {
        int j = idx[p];
        if (x[j] < kMinOcc) continue;
        double qq[6] = {q[3 * i], q[3 * i + 1], q[3 * i + 2],
                        q[3 * j], q[3 * j + 1], q[3 * j + 2]};
        double nn[2] = {x[i], x[j]};
        int sp[2] = {spc[i], spc[j]};
        acc += rho_F(nn, qq, sp);
      }
    }
    out[k] = acc;
  });
}

void orc_pt_DV_pairs(int n, const double *q, const double *x, const int *spc,
                     const double *rho, const int *offs, const int *idx, const int *u_list,
                     const int *i_list, int npairs, double *out3) {
  (void)n;
  View v{q, nullptr, x, rho, spc, offs, idx};
  par_for(npairs, [&](int k) { DV_dq(v, u_list[k], i_list[k], out3 + 3 * k); });
}

void orc_pt_DV_dF(int n, const double *q, const double *q0, const double *x, const int *spc,
                  const double *rho, const int *offs, const int *idx, const int *sites,
                  int nsites, double *out9) {
  (void)n;
  View v{q, nullptr, x, rho, spc, offs, idx};
  par_for(nsites, [&](int k) { DV_dF(v, q0, sites[k], out9 + 9 * k); });
}

void orc_mf_DV0_dF(int n, const double *q, const double *q0, const double *sigma,
                   const double *x, const int *spc, const double *rho, const int *offs,
                   const int *idx, const int *sites, int nsites, double *out9) {
  (void)n;
  View v{q, sigma, x, rho, spc, offs, idx};
  par_for(nsites, [&](int k) { DV0_dF(v, q0, sites[k], out9 + 9 * k); });
}

void orc_pt_D2V_pairs(int n, const double *q, const double *x, const int *spc,
                      const double *rho, const int *offs, const int *idx, const int *u_list,
                      const int *i_list, int npairs, double *out9) {
  (void)n;
  View v{q, nullptr, x, rho, spc, offs, idx};
  par_for(npairs, [&](int k) { D2V_dq2(v, u_list[k], i_list[k], out9 + 9 * k); });
}

void orc_mf_D2V0_pairs(int n, const double *q, const double *sigma, const double *x,
                       const int *spc, const double *rho, const int *offs, const int *idx,
                       const int *u_list, const int *i_list, int npairs, double *out9) {
  (void)n;
  View v{q, sigma, x, rho, spc, offs, idx};
  par_for(npairs, [&](int k) { D2V0_dq2(v, u_list[k], i_list[k], out9 + 9 * k); });
}

void orc_residuals(int n, const double *q, const double *sigma,
                   const double *x, const int *spc, const double *beta,
                   const double *gamma, const double *rho, const int *owner,
                   const int *image, const int *offs, const int *idx,
                   const int *u_list, int nu, double *Rq, double *Rs,
                   double *Rx) {
  (void)n;
  View v{q, sigma, x, rho, spc, offs, idx};
  par_for(nu, [&](int k) {
    int u = u_list[k];
    double rq[3] = {0, 0, 0}, rs = 0, rx = 0;
    if (!(x[u] < kMinOcc)) {
      // centres: u itself, then every neighbour of u (real or image)
      int ncen = 1 + offs[u + 1] - offs[u];
      for (int c = 0; c < ncen; ++c) {
        int ic = c == 0 ? u : idx[offs[u] + c - 1];
        int o = owner[ic];
        const int *T = image + 3 * ic;
        int uu = u;  // u as seen from the owner's frame
        if (T[0] != 0 || T[1] != 0 || T[2] != 0) {
          uu = -1;
          for (int p = offs[o]; p < offs[o + 1]; ++p) {
            int cand = idx[p];
            const int *Tc = image + 3 * cand;
            if (owner[cand] == u && Tc[0] == -T[0] && Tc[1] == -T[1] &&
                Tc[2] == -T[2]) {
              uu = cand;
              break;
            }
          }
          if (uu < 0) continue;  // pair straddles rc by rounding only
        }
        double g4[4];
        DV0_dq(v, uu, o, g4);
        double gx = DV0_dx(v, uu, o);
        double wgt = beta[o] / beta[u];
        for (int a = 0; a < 3; ++a) rq[a] += wgt * g4[a];
        rs += wgt * g4[3];
        rx += wgt * gx;
      }
      rs -= 3.0 / (beta[u] * sigma[u]);
      if (spc[u] == kH) {
        double xu = x[u];
        double dlogz = 3.0 / (2.0 * xu) + (xu < 1.0 ? 1.0 / (1.0 - xu) : 0.0);
        rx -= dlogz / beta[u];
        if (xu < 0.9999) rx -= gamma[u] / beta[u];
      } else {
        rx = 0.0;
      }
    }
    for (int a = 0; a < 3; ++a) Rq[3 * k + a] = rq[a];
    Rs[k] = rs;
    Rx[k] = rx;
  });
}

// Hydrogen master-equation update (project definition; the reference keeps
// only the parameters, Variables.hpp:68-92).  Sequential restatement of
// btam_dmd_step's integer update.
// Diffusive activity and degrees of the real H sites (shared by the update
// and the step-control decision).
static void orc_dmd_active(int n, const int *code_all, const int *owner, const double *x_all,
                           const int *moffs, const int *midx, const int *doffs,
                           const int *didx, const long long *X, std::vector<int> &active,
                           std::vector<long long> &deg) {
  const double q = 8.8817841970012523e-16;
  active.assign(n, 0);
  deg.assign(n, 0);
  // diffusive activity: x_i plus the occupancy of its H mechanical
  // neighbours reaches 0.01 (list_of_active_diffusive_sites_MgHx,
  // Topology.cpp:202-364)
  for (int i = 0; i < n; ++i) {
    if (code_all[i] != 1) continue;
    double mass = (double)X[i] * q;
    for (int p = moffs[i]; p < moffs[i + 1]; ++p)
      if (code_all[midx[p]] == 1) mass += x_all[midx[p]];
    active[i] = mass >= 0.01;
  }
  for (int i = 0; i < n; ++i)
    if (active[i])
      for (int p = doffs[i]; p < doffs[i + 1]; ++p) deg[i] += active[owner[didx[p]]];
}

// The room of edge (i, o) in quanta under the degree split.
static void orc_dmd_room(const long long *X, const std::vector<long long> &deg, int i, int o,
                         long long xmax, long long &hi, long long &lo) {
  long long di = deg[i] > 0 ? deg[i] : 1, dq = deg[o] > 0 ? deg[o] : 1;
  long long out_i = X[i] / di, out_o = X[o] / dq;
  long long in_i = xmax > X[i] ? (xmax - X[i]) / di : 0;
  long long in_o = xmax > X[o] ? (xmax - X[o]) / dq : 0;
  hi = out_i < in_o ? out_i : in_o;
  lo = -(out_o < in_i ? out_o : in_i);
}

// A move in quanta (v = the move times 2^50), rounded to nearest from a
// value first held within +-4e18, so that a move whose quanta overflow 64
// bits is cut to the edge's room like any other large move.
long long orc_dmd_quanta(double v) { return llrint(std::fmin(std::fmax(v, -4e18), 4e18)); }

void orc_dmd_control(int n, const int *code_all, const int *owner, const double *x_all,
                     const double *beta, const double *mu, const int *moffs, const int *midx,
                     const int *doffs, const int *didx, const double *params, double max_dx,
                     const long long *X, double *out2) {
  const double q = 8.8817841970012523e-16, invq = 1125899906842624.0;
  const double dt = params[0], Df = params[1], dr = params[2], min_dx = params[3],
               max_x = params[4];
  std::vector<int> active;
  std::vector<long long> deg;
  orc_dmd_active(n, code_all, owner, x_all, moffs, midx, doffs, didx, X, active, deg);
  const long long xmax = llrint(max_x * invq);
  double ratio = 0.0, worst_dx = 0.0;
  for (int i = 0; i < n; ++i) {
    if (!active[i]) continue;
    double dx = 0.0;
    for (int p = doffs[i]; p < doffs[i + 1]; ++p) {
      int o = owner[didx[p]];
      if (o == i || !active[o]) continue;
      double xi = (double)X[i] * q, xo = (double)X[o] * q;
      double xm = 0.5 * (xi + xo), bm = 0.5 * (beta[i] + beta[o]);
      double J = Df / (dr * dr) * bm * xm * (1.0 - xm) * (mu[i] - mu[o]);
      double dlt = dt * J;
      if (std::fabs(dlt) < min_dx) continue;
      dx -= dlt;
      if (o < i) continue;
      long long qn = orc_dmd_quanta(dlt * invq), hi, lo;
      orc_dmd_room(X, deg, i, o, xmax, hi, lo);
      if (qn > hi && hi > 0) ratio = std::max(ratio, (double)qn / (double)hi);
      if (qn < lo && lo < 0) ratio = std::max(ratio, (double)qn / (double)lo);
    }
    worst_dx = std::max(worst_dx, std::fabs(dx) / max_dx);
  }
  out2[0] = ratio;
  out2[1] = worst_dx;
}

void orc_dmd_update(int n, const int *code_all, const int *owner, const double *x_all,
                    const double *beta, const double *mu, const int *moffs,
                    const int *midx, const int *doffs, const int *didx,
                    const double *params, long long *X, long long *clipped) {
  const double q = 8.8817841970012523e-16, invq = 1125899906842624.0;
  const double dt = params[0], Df = params[1], dr = params[2], min_dx = params[3],
               max_x = params[4];
  std::vector<int> active;
  std::vector<long long> deg, X0(X, X + n);
  orc_dmd_active(n, code_all, owner, x_all, moffs, midx, doffs, didx, X0.data(), active, deg);
  const long long xmax = llrint(max_x * invq);
  for (int i = 0; i < n; ++i) {
    if (!active[i]) continue;
    for (int p = doffs[i]; p < doffs[i + 1]; ++p) {
      int o = owner[didx[p]];
      if (o <= i || !active[o]) continue;
      double xi = (double)X0[i] * q, xo = (double)X0[o] * q;
      double xm = 0.5 * (xi + xo), bm = 0.5 * (beta[i] + beta[o]);
      double J = Df / (dr * dr) * bm * xm * (1.0 - xm) * (mu[i] - mu[o]);
      double dlt = dt * J;
      if (std::fabs(dlt) < min_dx) continue;
      long long qn = orc_dmd_quanta(dlt * invq), hi, lo;
      orc_dmd_room(X0.data(), deg, i, o, xmax, hi, lo);
      if (clipped && ((qn > hi && hi > 0) || (qn < lo && lo < 0))) ++*clipped;
      qn = qn > hi ? hi : (qn < lo ? lo : qn);
      X[i] -= qn;
      X[o] += qn;
    }
  }
}

// The 5th-degree rule over the pair measure (Quadrature-Hermitian-5th.cpp:
// 31-432) of pair term `term` (0 rho, 1 pair): mode 0 the average of F,
// 1 of dF_dq(direction), 2 of d2F_dq2(direction) (a pair's blocks: 0 and 3
// the Hessian H of the radial term, 1 and 2 -H).  44 points, the 22 of the
// table and their negatives: z = (1, ..., 1) with weight 1/128, sqrt(2)
// e_k (k = 0..5) with weight 1/16, and (1, ..., 1) with two entries -1
// (pairs a < b in order) with weight 1/128; q = mean +- sqrt(2) sigma_s z
// (sigma of the site of each coordinate); each value weighted W c0,
// c0 = pi^(3/2), the sum scaled by pi^(-3/2).
int orc_quad5(int term, int mode, int direction, const double *q, const double *sigma,
              const double *x, const int *spc, double *out) {
  if (term < 0 || term > 1 || mode < 0 || mode > 2) return 1;
  const Term &t = term == 0 ? kRho : kPair;
  const double s2 = 1.4142135623730951, PI = 3.14159265358979323846;
  double z[22][6], W[22];
  for (int k = 0; k < 6; ++k) z[0][k] = 1.0;
  W[0] = 0.0078125;
  for (int g = 1; g <= 6; ++g) {
    for (int k = 0; k < 6; ++k) z[g][k] = k == g - 1 ? s2 : 0.0;
    W[g] = 0.0625;
  }
  int g = 7;
  for (int a = 0; a < 6; ++a)
    for (int b = a + 1; b < 6; ++b, ++g) {
      for (int k = 0; k < 6; ++k) z[g][k] = (k == a || k == b) ? -1.0 : 1.0;
      W[g] = 0.0078125;
    }
  const double c0 = std::pow(std::sqrt(PI), 6.0 / 2.0);
  const int nv = mode == 0 ? 1 : mode == 1 ? 3 : 9;
  for (int e = 0; e < 9; ++e) out[e] = 0.0;
  for (int sg = 0; sg < 2; ++sg)
    for (int gp = 0; gp < 22; ++gp) {
      double ql[6], v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int a = 0; a < 3; ++a)
        for (int s = 0; s < 2; ++s) {
          const double off = s2 * sigma[s] * z[gp][s * 3 + a];
          ql[s * 3 + a] = sg == 0 ? q[s * 3 + a] + off : q[s * 3 + a] - off;
        }
      if (mode == 0) {
        v[0] = t.F(x, ql, spc);
      } else if (mode == 1) {
        t.dq(direction, v, x, ql, spc);
      } else {
        term_d2(term, 0, x, ql, spc, v);
        if (direction == 1 || direction == 2)
          for (int e = 0; e < 9; ++e) v[e] = -v[e];
      }
      for (int e = 0; e < nv; ++e) out[e] += v[e] * W[gp] * c0;
    }
  for (int e = 0; e < nv; ++e) out[e] = out[e] * std::pow(1.0 / std::sqrt(PI), 6.0 / 2.0);
  return 0;
}

// One slot of the reference's per-term table (potential_function,
// Macros.hpp:252-278) at one geometry: fn 0 F, 1 dF_dq, 2 d2F_dq2 (the
// diagonal blocks a (ns + 1) only; other blocks return 1), 3 dF_dq_FD
// (d_rho_ij_dq_FD, MgHx-ADP.cpp:605-661, and its three twins: five points,
// step 1e-4, 1e-5 for the pair term, the moved coordinate left at +2 dr
// while the next one moves), 4 d2F_dq2_FD (736-812: the diagonal of the
// slot direction / (ns + 1)),
// 5 dF_dn.  out: 9 values, unused ones 0.
int orc_term_eval(int term, int fn, int dir, int ns, const double *q, const double *x,
                  const int *spc, double *out) {
  const Term *t = term == 0 ? &kRho : term == 1 ? &kPair : term == 2 ? &kDip
                : term == 3 ? &kQuad : nullptr;
  if (!t || ns != (term < 2 ? 2 : 3)) return 1;
  for (int e = 0; e < 9; ++e) out[e] = 0.0;
  const double dr = 0.0001;
  if (fn == 0) {
    out[0] = t->F(x, q, spc);
  } else if (fn == 1) {
    t->dq(dir, out, x, q, spc);
  } else if (fn == 2) {
    if (dir % (ns + 1) != 0) return 1;
    term_d2(term, dir / (ns + 1), x, q, spc, out);
  } else if (fn == 3) {
    // the pair term's twin steps by 1e-5 (dV_pair_ij_dq_FD, 953-1008)
    const double h = term == 1 ? 0.00001 : dr;
    const double f0 = t->F(x, q, spc);
    double qn[9];
    for (int e = 0; e < 3 * ns; ++e) qn[e] = q[e];
    for (int a = 0; a < 3; ++a) {
      const int d = 3 * dir + a;
      qn[d] = q[d] - h * 2;
      const double fmm = t->F(x, qn, spc);
      qn[d] = q[d] - h;
      const double fm = t->F(x, qn, spc);
      qn[d] = q[d] + h;
      const double fp = t->F(x, qn, spc);
      qn[d] = q[d] + h * 2;
      const double fpp = t->F(x, qn, spc);
      out[a] = ((fmm - f0) - 8.0 * (fm - f0) + 8.0 * (fp - f0) - (fpp - f0)) / (12.0 * h);
    }
  } else if (fn == 4) {
    // the quadrupole's fills the diagonal blocks 0, 4 and 8 only
    // (dV2_quadrupole_ij1j2_dq2_FD, 2270-2349)
    if (term == 3 && dir % (ns + 1) != 0) return 0;
    const double f0 = t->F(x, q, spc);
    for (int a = 0; a < 3; ++a) {
      const int d = dir / (1 + ns) * 3 + a;
      double qs[4][9], f[4];
      for (int w = 0; w < 4; ++w) {
        for (int e = 0; e < 3 * ns; ++e) qs[w][e] = q[e];
        const double D = 1.0;
        qs[w][d] = w == 0 ? q[d] + D * dr * 2 : w == 1 ? q[d] + D * dr
                 : w == 2 ? q[d] - D * dr : q[d] - D * dr * 2;
        f[w] = t->F(x, qs[w], spc);
      }
      out[4 * a] = (-f[0] + 16.0 * f[1] - 30.0 * f0 + 16.0 * f[2] - f[3]) / (12.0 * dr * dr);
    }
  } else if (fn == 5) {
    out[0] = t->dn(dir, x, q, spc);
  } else {
    return 1;
  }
  return 0;
}

}  // extern "C"
