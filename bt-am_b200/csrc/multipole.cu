// Mean-field energy forms under the multipole rule: the reference's
// alternative to the degree-3 Gauss-Hermite rule behind its compile switch
// (MULTIPOLE_INTEGRAL, MgHx-mf-V-bulk.cpp:715-724;
// meanfield_integral_mp, Quadrature-Multipole.cpp:97-143):
//   <f> = f(mean) + sum_{(a, b) in dof} sigma_a^2 / 2 tr d2f/dq_a dq_b,
// with the pair measure's dof table {(0,0), (1,1)} and the triplet
// measure's {(0,0), (1,1), (2,2)} plus (1,2), (2,1) when j1 = j2
// (MgHx-mf-V-bulk.cpp:890-895).  Two Hessian variants:
//   rule 1, as the reference's build flags compile it: CMakeLists.txt:185
//     defines NUMERICAL_DERIVATIVES=0, and `#ifdef` (Quadrature-
//     Multipole.cpp:134) then selects the finite-difference Hessians
//     (MgHx-ADP.cpp:736-812, 1091-1167, 1605-1680, 2270-2349): only the
//     diagonal entries, each a five-point second difference with step 1e-4
//     along coordinate al of slot direction / (ns + 1).  The dipole's
//     j1-j2 directions 5 and 7 thus repeat slot 1; the quadrupole's give
//     zero.  These kernels restate the energy functions in the reference's
//     operation order, and this file is compiled without FMA contraction,
//     so each term's value is the reference's to the last bit, which the
//     1/(12 dr^2) = 8.3e6 of the second difference would otherwise amplify;
//   rule 2, NUMERICAL_DERIVATIVES undefined: the analytic Hessians'
//     traces, in closed form (Laplacians of the radial, vector and tensor
//     terms).
// The evaluation is direct, not through moments: a warp per real site;
// lanes over its list entries (rho-bar, pair terms) and over the j1 <= j2
// triangle of its list (triplet terms), FP64.  Rule 1 evaluates each
// triplet at 37 geometries.  No solver of the reference runs this rule in
// its shipped build; it is here for the callers that select it.
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace btam {
double tables_mass(const btam_tables *t, int code);
namespace {

constexpr double kSqrt2d = 1.4142135623730951;  // sqrt(2) of the rule (Macros.hpp)

// cubic_spline (cubic-spline.cpp:84-96) in the reference's operation order:
// m = min((int)(x / dx), n - 1), p = min(x - m dx, dx); a negative x (an
// embedding density below 0) takes segment 0 instead of an index before
// the table.
__device__ __forceinline__ int seg_ref(double x, double dx, int n, double &p) {
  int m = (int)(x / dx);
  m = m < n - 1 ? m : n - 1;
  m = m > 0 ? m : 0;
  p = (double)m * dx;
  p = x - p;
  p = fmin(p, dx);
  return m;
}
__device__ __forceinline__ double cubv(const double *k, double p) {
  return k[0] + (k[1] + (k[2] + k[3] * p) * p) * p;
}
// d_cubic_spline: b + (2c + 3d p) p, with the reference's db/dc/dd columns
// (b, 2c, 3d).
__device__ __forceinline__ double cubd(const double *k, double p) {
  return k[1] + (2.0 * k[2] + 3.0 * k[3] * p) * p;
}
__device__ __forceinline__ double cubdd(const double *k, double p) {
  return 2.0 * k[2] + 6.0 * k[3] * p;
}
__device__ __forceinline__ double tab_v(const SplineView<double> &S, double x) {
  double p;
  const int m = seg_ref(x, S.dx, S.n, p);
  const Coef4<double> c = S.c[m];
  return c.a + (c.b + (c.c + c.d * p) * p) * p;
}

__device__ __forceinline__ double sqz(double a) { return a == 0.0 ? 0.0 : a * a; }  // DSQR

// rho_ij (MgHx-ADP.cpp:526-553): n_j rho_{s_j}(|q_i - q_j|).
__device__ __forceinline__ double rho_F(const RadialView<double> &T, int pk, int cj, double nj,
                                        const double *q) {
  double r2 = 0.0;
  for (int a = 0; a < 3; ++a) r2 += sqz(q[a] - q[3 + a]);
  double p;
  const int m = seg_ref(sqrt(r2), T.dx, T.n, p);
  return nj * cubv(pr_rec(T, pk, m) + rho_off(pk, cj), p);
}
// V_pair_ij (869-900): 1/2 n_i n_j phi(|q_i - q_j|).
__device__ __forceinline__ double pair_F(const RadialView<double> &T, int pk, double ni,
                                         double nj, const double *q) {
  double r2 = 0.0;
  for (int a = 0; a < 3; ++a) r2 += sqz(q[a] - q[3 + a]);
  double p;
  const int m = seg_ref(sqrt(r2), T.dx, T.n, p);
  const double phi = ni * nj * cubv(pr_rec(T, pk, m), p);
  return 0.5 * phi;
}
// V_dipole_ij1j2 (1233-1281) and V_quadrupole_ij1j2 (1781-1831) at one
// geometry q = (q_i, q_j1, q_j2).
__device__ __forceinline__ void tri_F(const RadialView<double> &T, int pk1, int pk2,
                                      const double *n, const double *q, double &fd,
                                      double &fq) {
  double r1sq = 0.0, r2sq = 0.0, dot = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double r1 = q[a] - q[3 + a], r2 = q[a] - q[6 + a];
    r1sq += sqz(r1);
    r2sq += sqz(r2);
    dot += r1 * r2;
  }
  double p1, p2;
  const int m1 = seg_ref(sqrt(r1sq), T.dx, T.n, p1);
  const int m2 = seg_ref(sqrt(r2sq), T.dx, T.n, p2);
  double k1[8], k2[8];
  ld8(uw_rec(T, pk1, m1), k1);
  ld8(uw_rec(T, pk2, m2), k2);
  const double u1 = n[0] * n[1] * cubv(k1, p1), u2 = n[0] * n[2] * cubv(k2, p2);
  const double w1 = n[0] * n[1] * cubv(k1 + 4, p1), w2 = n[0] * n[2] * cubv(k2 + 4, p2);
  fd = (1.0 / 2.0) * u1 * u2 * dot;
  fq = (1.0 / 2.0) * w1 * w2 * sqz(dot) - (1.0 / 6.0) * w1 * w2 * r1sq * r2sq;
}

// The five-point second difference (step 1e-4) of the FD Hessians.
__device__ __forceinline__ double d2_5(double fpp, double fp, double f0, double fm, double fmm) {
  const double dr = 0.0001;
  return (-fpp + 16.0 * fp - 30.0 * f0 + 16.0 * fm - fmm) / (12.0 * dr * dr);
}

// Coordinates moved as the FD Hessians move them: q + D dr 2, q + D dr,
// q - D dr, q - D dr 2 with D = 1 on coordinate k only.
template <int N>
__device__ __forceinline__ void shifted(const double (&q)[N], int k, int which, double (&o)[N]) {
  const double dr = 0.0001;
#pragma unroll
  for (int c = 0; c < N; ++c) {
    const double D = c == k ? 1.0 : 0.0;
    o[c] = which == 0 ? q[c] + D * dr * 2 : which == 1 ? q[c] + D * dr
                                         : which == 2 ? q[c] - D * dr
                                                      : q[c] - D * dr * 2;
  }
}

struct PairSite {
  double q[3], sig, x;
  int code;
};

// Multipole average of rho_ij (term 0) or V_pair_ij (term 1) over the pair
// measure (i, j).
__device__ double pair_mp(const RadialView<double> &T, int rule, int term, const PairSite &i,
                          const PairSite &j) {
  const int pk = pair_kind(i.code, j.code);
  const double q[6] = {i.q[0], i.q[1], i.q[2], j.q[0], j.q[1], j.q[2]};
  auto F = [&](const double (&qq)[6]) {
    return term == 0 ? rho_F(T, pk, j.code, j.x, qq) : pair_F(T, pk, i.x, j.x, qq);
  };
  const double f0 = F(q);
  double acc = f0;
  if (rule == 1) {
    for (int a = 0; a < 2; ++a) {
      const double c2 = sqz(a == 0 ? i.sig : j.sig) / 2.0;
      for (int al = 0; al < 3; ++al) {
        double s[4];
        for (int w = 0; w < 4; ++w) {
          double qq[6];
          shifted(q, 3 * a + al, w, qq);
          s[w] = F(qq);
        }
        acc += c2 * d2_5(s[0], s[1], f0, s[2], s[3]);
      }
    }
  } else {
    // tr of both diagonal blocks: g'' + 2 g' / s (n_j rho or 1/2 n_i n_j phi)
    double r2 = 0.0;
    for (int a = 0; a < 3; ++a) r2 += sqz(q[a] - q[3 + a]);
    const double s = sqrt(r2);
    double p;
    const int m = seg_ref(s, T.dx, T.n, p);
    const double *k = term == 0 ? pr_rec(T, pk, m) + rho_off(pk, j.code) : pr_rec(T, pk, m);
    const double c = term == 0 ? j.x : 0.5 * i.x * j.x;
    const double lap = c * (cubdd(k, p) + 2.0 * cubd(k, p) / s);
    acc += sqz(i.sig) / 2.0 * lap;
    acc += sqz(j.sig) / 2.0 * lap;
  }
  return acc;
}

// Closed-form traces of the triplet Hessian blocks (rule 2).  With
// r_k = q_i - q_jk, s_k = |r_k|, d = r1.r2, c_k = n_i n_jk, spline values
// u, w and derivatives ', '':
//   dipole 1/2 c1 c2 u1 u2 d:
//     slot 1 alone   1/2 c1 c2 u2 d (u1'' + 4 u1' / s1)
//     cross (1, 2)   1/2 c1 c2 (u1' u2' d^2 / (s1 s2) + u1' u2 s1 + u1 u2' s2 + 3 u1 u2)
//   quadrupole c1 c2 (1/2 w1 w2 d^2 - 1/6 w1 w2 s1^2 s2^2):
//     slot 1 alone   c1 c2 (1/2 w2 ((w1'' + 6 w1'/s1) d^2 + 2 w1 s2^2)
//                           - 1/6 w2 s2^2 (w1'' s1^2 + 6 w1' s1 + 6 w1))
//     cross (1, 2)   1/2 c1 c2 d (w1' w2' d^2/(s1 s2) + 2 w1' w2 s1 + 2 w1 w2' s2 + 8 w1 w2)
//                    - 1/6 c1 c2 d (w1' s1 + 2 w1)(w2' s2 + 2 w2)
//   and the centre block (q_i moves both r_k) is slot 1 + slot 2 + 2 cross.
struct TriTr {
  double d11, d22, d12, q11, q22, q12;
};
__device__ __forceinline__ TriTr tri_traces(const RadialView<double> &T, int pk1, int pk2, const double *n,
                            const double *q) {
  double r1sq = 0.0, r2sq = 0.0, d = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double r1 = q[a] - q[3 + a], r2 = q[a] - q[6 + a];
    r1sq += sqz(r1);
    r2sq += sqz(r2);
    d += r1 * r2;
  }
  const double s1 = sqrt(r1sq), s2 = sqrt(r2sq);
  double p1, p2;
  const int m1 = seg_ref(s1, T.dx, T.n, p1), m2 = seg_ref(s2, T.dx, T.n, p2);
  double k1[8], k2[8];
  ld8(uw_rec(T, pk1, m1), k1);
  ld8(uw_rec(T, pk2, m2), k2);
  const double c = (n[0] * n[1]) * (n[0] * n[2]);
  const double u1 = cubv(k1, p1), du1 = cubd(k1, p1), ddu1 = cubdd(k1, p1);
  const double u2 = cubv(k2, p2), du2 = cubd(k2, p2), ddu2 = cubdd(k2, p2);
  const double w1 = cubv(k1 + 4, p1), dw1 = cubd(k1 + 4, p1), ddw1 = cubdd(k1 + 4, p1);
  const double w2 = cubv(k2 + 4, p2), dw2 = cubd(k2 + 4, p2), ddw2 = cubdd(k2 + 4, p2);
  TriTr t;
  t.d11 = 0.5 * c * u2 * d * (ddu1 + 4.0 * du1 / s1);
  t.d22 = 0.5 * c * u1 * d * (ddu2 + 4.0 * du2 / s2);
  t.d12 = 0.5 * c * (du1 * du2 * d * d / (s1 * s2) + du1 * u2 * s1 + u1 * du2 * s2 + 3.0 * u1 * u2);
  t.q11 = c * (0.5 * w2 * ((ddw1 + 6.0 * dw1 / s1) * d * d + 2.0 * w1 * r2sq) -
               w2 * r2sq * (ddw1 * r1sq + 6.0 * dw1 * s1 + 6.0 * w1) / 6.0);
  t.q22 = c * (0.5 * w1 * ((ddw2 + 6.0 * dw2 / s2) * d * d + 2.0 * w2 * r1sq) -
               w1 * r1sq * (ddw2 * r2sq + 6.0 * dw2 * s2 + 6.0 * w2) / 6.0);
  t.q12 = 0.5 * c * d *
              (dw1 * dw2 * d * d / (s1 * s2) + 2.0 * dw1 * w2 * s1 + 2.0 * w1 * dw2 * s2 +
               8.0 * w1 * w2) -
          c * d * (dw1 * s1 + 2.0 * w1) * (dw2 * s2 + 2.0 * w2) / 6.0;
  return t;
}

// Multipole averages of V_dipole and V_quadrupole over the triplet measure
// (i, j1, j2) (meanfield_integral_mp on the measures of
// MgHx-mf-V-bulk.cpp:897-932).
__device__ void tri_mp(const RadialView<double> &T, int rule, const PairSite &i,
                       const PairSite &j1, const PairSite &j2, bool coincident, double &vd,
                       double &vq) {
  const int pk1 = pair_kind(i.code, j1.code), pk2 = pair_kind(i.code, j2.code);
  const double n[3] = {i.x, j1.x, j2.x};
  const double q[9] = {i.q[0],  i.q[1],  i.q[2],  j1.q[0], j1.q[1],
                       j1.q[2], j2.q[0], j2.q[1], j2.q[2]};
  const double sig[3] = {i.sig, j1.sig, j2.sig};
  double f0d, f0q;
  tri_F(T, pk1, pk2, n, q, f0d, f0q);
  vd = f0d;
  vq = f0q;
  if (rule == 1) {
    // second differences of slot `slot` along each axis (dipole, quadrupole)
    double fdd[3][3], fdq[3][3];
    for (int slot = 0; slot < 3; ++slot)
      for (int al = 0; al < 3; ++al) {
        double sd[4], sq4[4];
        for (int w = 0; w < 4; ++w) {
          double qq[9];
          shifted(q, 3 * slot + al, w, qq);
          tri_F(T, pk1, pk2, n, qq, sd[w], sq4[w]);
        }
        fdd[slot][al] = d2_5(sd[0], sd[1], f0d, sd[2], sd[3]);
        fdq[slot][al] = d2_5(sq4[0], sq4[1], f0q, sq4[2], sq4[3]);
      }
    // rows a = 0, 1, 2 of the dof table, in the reference's (a, b) order;
    // direction a * 3 + b reads slot (a * 3 + b) / 4
    for (int a = 0; a < 3; ++a) {
      const double c2 = sqz(sig[a]) / 2.0;
      for (int b = 0; b < 3; ++b) {
        if (!(a == b || (coincident && a > 0 && b > 0))) continue;
        const int dir = a * 3 + b, slot = dir / 4;
        const bool diag = dir == 0 || dir == 4 || dir == 8;
        for (int al = 0; al < 3; ++al) {
          vd += c2 * fdd[slot][al];
          if (diag) vq += c2 * fdq[slot][al];
        }
      }
    }
  } else {
    const TriTr t = tri_traces(T, pk1, pk2, n, q);
    const double c0 = sqz(sig[0]) / 2.0, c1 = sqz(sig[1]) / 2.0, c2 = sqz(sig[2]) / 2.0;
    vd += c0 * (t.d11 + t.d22 + 2.0 * t.d12);
    vq += c0 * (t.q11 + t.q22 + 2.0 * t.q12);
    vd += c1 * t.d11;
    vq += c1 * t.q11;
    if (coincident) {
      vd += c1 * t.d12;
      vq += c1 * t.q12;
      vd += c2 * t.d12;
      vq += c2 * t.q12;
    }
    vd += c2 * t.d22;
    vq += c2 * t.q22;
  }
}

struct MpArgs {
  int n_real, rule;
  const double4 *pos;  // q, sigma
  const double2 *xb;
  const int *code, *offs, *idx;
  RadialView<double> T;
  SplineView<double> emb_mg, emb_h;
  const double *rho;  // multipole rho-bar of the real sites (V0 kernel)
  double *out;
  double *S0;             // V0 kernel: the free entropy as well (may be null)
  const double *gamma;    // per real site
  double mass[2];         // Mg, H
};

__device__ __forceinline__ PairSite site_of(const MpArgs &a, int j) {
  const double4 p = a.pos[j];
  PairSite s;
  s.q[0] = p.x;
  s.q[1] = p.y;
  s.q[2] = p.z;
  s.sig = p.w;
  s.x = a.xb[j].x;
  s.code = a.code[j];
  return s;
}
// The site tests of the reference: H with x below min_occupancy is empty.
__device__ __forceinline__ bool empty_h(const PairSite &s) {
  return s.code == 1 && s.x < kMinOcc;
}

// evaluate_mf_rho_i_adp_MgHx (MgHx-mf-V-bulk.cpp:708-787) under the rule.
__global__ void __launch_bounds__(128) mp_rho_kernel(MpArgs a) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.n_real) return;
  const PairSite si = site_of(a, i);
  double acc = 0.0;
  if (!empty_h(si))
    for (int k = a.offs[i] + lane; k < a.offs[i + 1]; k += 32) {
      const PairSite sj = site_of(a, a.idx[k]);
      if (empty_h(sj)) continue;
      acc += pair_mp(a.T, a.rule, 0, si, sj);
    }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) a.out[i] = acc;
}

// evaluate_V0_i_adp_MgHx (791-953) under the rule: x_i F(rho-bar_i) plus the
// pair terms (j1 not an empty H) and the triplet terms (j1 <= j2 in the
// list, j2 of any species with x >= min_occupancy, factor 2 for j1 < j2).
// Lanes take the pair terms by list entry and the triplets by their index
// in the j1 <= j2 triangle.
__global__ void __launch_bounds__(128) mp_v0_kernel(MpArgs a) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.n_real) return;
  const PairSite si = site_of(a, i);
  const int nb0 = a.offs[i], nn = a.offs[i + 1] - nb0;
  double pair = 0.0, dip = 0.0, quad = 0.0;
  if (!empty_h(si)) {
    for (int k = lane; k < nn; k += 32) {
      const PairSite sj = site_of(a, a.idx[nb0 + k]);
      if (empty_h(sj)) continue;
      pair += pair_mp(a.T, a.rule, 1, si, sj);
    }
    const long long ntri = (long long)nn * (nn + 1) / 2;
    for (long long t = lane; t < ntri; t += 32) {
      // t = k2 (k2 + 1) / 2 + k1 with k1 <= k2
      int k2 = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
      while ((long long)k2 * (k2 + 1) / 2 > t) --k2;
      while ((long long)(k2 + 1) * (k2 + 2) / 2 <= t) ++k2;
      const int k1 = (int)(t - (long long)k2 * (k2 + 1) / 2);
      const PairSite s1 = site_of(a, a.idx[nb0 + k1]);
      if (empty_h(s1)) continue;
      const PairSite s2 = site_of(a, a.idx[nb0 + k2]);
      if (s2.x < kMinOcc) continue;
      double vd, vq;
      tri_mp(a.T, a.rule, si, s1, s2, k1 == k2, vd, vq);
      const double f = k1 == k2 ? 1.0 : 2.0;
      dip += f * vd;
      quad += f * vq;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    pair += __shfl_xor_sync(0xffffffffu, pair, off);
    dip += __shfl_xor_sync(0xffffffffu, dip, off);
    quad += __shfl_xor_sync(0xffffffffu, quad, off);
  }
  if (lane == 0) {
    double v = 0.0;
    if (!empty_h(si)) {
      const double emb = si.x * tab_v(si.code == 0 ? a.emb_mg : a.emb_h, a.rho[i]);
      v = emb + pair + dip + quad;
    }
    a.out[i] = v;
    if (a.S0) {
      // evaluate_S0_i_adp_MgHx (957-1142) on this V0: -log Z0 + beta H0 -
      // gamma x~, H0 = 1 / (2 beta) + V0; zero for x below min_occupancy
      double S = 0.0;
      if (!(si.x < kMinOcc)) {
        const double beta = a.xb[i].y;
        const double m = kUma * si.x * a.mass[si.code];
        double logZ = 3.0 * log((si.sig * sqrt(m / beta)) / kHbar);
        if (si.x < 1.0) logZ += log(1.0 / (1.0 - si.x));
        const double gx = si.code == 1 ? a.gamma[i] * (si.x > 0.9999 ? 0.9999 : si.x) : 0.0;
        S = -logZ + beta * (1.0 / (2.0 * beta) + v) - gx;
      }
      a.S0[i] = S;
    }
  }
}

// ---- residuals under the rule ---------------------------------------------
// The residual kernel calls its geometry functions out of line: inlined
// into every step of the unrolled second differences they overflow the
// instruction cache (the kernel stalled on instruction fetch).  The
// energy kernels keep them inline.  Rounding is the same either way.
__device__ __noinline__ double rho_F_call(const RadialView<double> &T, int pk, int cj, double nj,
                                          const double *q) {
  return rho_F(T, pk, cj, nj, q);
}
__device__ __noinline__ double pair_F_call(const RadialView<double> &T, int pk, double ni,
                                           double nj, const double *q) {
  return pair_F(T, pk, ni, nj, q);
}
__device__ __noinline__ void tri_F_call(const RadialView<double> &T, int pk1, int pk2,
                                        const double *n, const double *q, double &fd,
                                        double &fq) {
  tri_F(T, pk1, pk2, n, q, fd, fq);
}
__device__ __noinline__ TriTr tri_traces_call(const RadialView<double> &T, int pk1, int pk2,
                                              const double *n, const double *q) {
  return tri_traces(T, pk1, pk2, n, q);
}
// evaluate_DV0_i_Dq_u_MgHx (MgHx-mf-V-bulk.cpp:1823-2098) with
// meanfield_integral_mp_dmq / _dsq (Quadrature-Multipole.cpp:147-286) and
// evaluate_DV0_i_Dxi_u_adp_MgHx (2102-2325), whose occupancy integrals stay
// on the degree-3 rule (meanfield_integral_gh_3th_dxi) at the multipole
// rho-bar.  Gradient and occupancy functions in the reference's operation
// order (MgHx-ADP.cpp:557-601, 815-844, 904-949, 1170-1209, 1285-1371,
// 1683-1758, 1835-1935, 2352-2434).

// d rho_ij / dq_dir (dir 0: q_i, 1: q_j).
__device__ __noinline__ void rho_dq(const RadialView<double> &T, int pk, int cj, double nj, int dir,
                       const double *q, double *out) {
  double r[3], r2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sqz(r[a]);
  }
  const double nr = sqrt(r2), inv = 1.0 / nr;
  double p;
  const int m = seg_ref(nr, T.dx, T.n, p);
  const double g = nj * cubd(pr_rec(T, pk, m) + rho_off(pk, cj), p);
  for (int a = 0; a < 3; ++a) out[a] = dir == 0 ? g * inv * r[a] : -g * inv * r[a];
}
__device__ __noinline__ void pair_dq(const RadialView<double> &T, int pk, double ni, double nj, int dir,
                        const double *q, double *out) {
  double r[3], r2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    r[a] = q[a] - q[3 + a];
    r2 += sqz(r[a]);
  }
  const double nr = sqrt(r2), inv = 1.0 / nr;
  double p;
  const int m = seg_ref(nr, T.dx, T.n, p);
  const double g = ni * nj * cubd(pr_rec(T, pk, m), p);
  for (int a = 0; a < 3; ++a) out[a] = dir == 0 ? 0.5 * g * inv * r[a] : -0.5 * g * inv * r[a];
}
// d V_dipole / dq_dir and d V_quadrupole / dq_dir at one geometry.
__device__ __noinline__ void tri_dq(const RadialView<double> &T, int pk1, int pk2, const double *n, int dir,
                       const double *q, double *gd, double *gq) {
  double r1[3], r2[3], r1sq = 0.0, r2sq = 0.0, dot = 0.0;
  for (int a = 0; a < 3; ++a) {
    r1[a] = q[a] - q[3 + a];
    r2[a] = q[a] - q[6 + a];
    r1sq += sqz(r1[a]);
    r2sq += sqz(r2[a]);
    dot += r1[a] * r2[a];
  }
  const double n1 = sqrt(r1sq), n2 = sqrt(r2sq);
  double p1, p2;
  const int m1 = seg_ref(n1, T.dx, T.n, p1), m2 = seg_ref(n2, T.dx, T.n, p2);
  double k1[8], k2[8];
  ld8(uw_rec(T, pk1, m1), k1);
  ld8(uw_rec(T, pk2, m2), k2);
  const double i1 = 1.0 / n1, i2 = 1.0 / n2;
  const double c1 = n[0] * n[1], c2 = n[0] * n[2];
  const double u1 = c1 * cubv(k1, p1), u2 = c2 * cubv(k2, p2);
  const double du1 = c1 * cubd(k1, p1), du2 = c2 * cubd(k2, p2);
  const double w1 = c1 * cubv(k1 + 4, p1), w2 = c2 * cubv(k2 + 4, p2);
  const double dw1 = c1 * cubd(k1 + 4, p1), dw2 = c2 * cubd(k2 + 4, p2);
  const double dd = sqz(dot);
  for (int a = 0; a < 3; ++a) {
    if (dir == 0) {
      gd[a] = 0.5 * (du1 * u2 * dot * i1 * r1[a] + u1 * du2 * dot * i2 * r2[a] +
                     u1 * u2 * (r1[a] + r2[a]));
      gq[a] = (1.0 / 2.0) * (dw1 * w2 * dd * i1 * r1[a] + w1 * dw2 * dd * i2 * r2[a] +
                             w1 * w2 * 2 * dot * (r1[a] + r2[a])) -
              (1.0 / 6.0) * (dw1 * w2 * n1 * r2sq * r1[a] + w1 * dw2 * r1sq * n2 * r2[a] +
                             w1 * w2 * 2 * r2sq * r1[a] + w1 * w2 * 2 * r1sq * r2[a]);
    } else if (dir == 1) {
      gd[a] = -0.5 * (du1 * u2 * dot * i1 * r1[a] + u1 * u2 * r2[a]);
      gq[a] = -0.5 * (dw1 * w2 * dd * i1 * r1[a] + w1 * w2 * 2 * dot * r2[a]) +
              (1.0 / 6.0) * (dw1 * w2 * n1 * r2sq * r1[a] + w1 * w2 * 2 * r2sq * r1[a]);
    } else {
      gd[a] = -0.5 * (u1 * du2 * dot * i2 * r2[a] + u1 * u2 * r1[a]);
      gq[a] = -0.5 * (w1 * dw2 * dd * i2 * r2[a] + w1 * w2 * 2 * dot * r1[a]) +
              (1.0 / 6.0) * (w1 * dw2 * r1sq * n2 * r2[a] + w1 * w2 * 2 * r1sq * r2[a]);
    }
  }
}
// d / dn_dir of the four terms (occupancy derivatives).
__device__ __noinline__ double rho_dn(const RadialView<double> &T, int pk, int cj, int dir, const double *q) {
  if (dir != 1) return 0.0;
  double r2 = 0.0;
  for (int a = 0; a < 3; ++a) r2 += sqz(q[a] - q[3 + a]);
  double p;
  const int m = seg_ref(sqrt(r2), T.dx, T.n, p);
  return cubv(pr_rec(T, pk, m) + rho_off(pk, cj), p);
}
__device__ __noinline__ double pair_dn(const RadialView<double> &T, int pk, const double *n, int dir,
                          const double *q) {
  double r2 = 0.0;
  for (int a = 0; a < 3; ++a) r2 += sqz(q[a] - q[3 + a]);
  double p;
  const int m = seg_ref(sqrt(r2), T.dx, T.n, p);
  const double phi = cubv(pr_rec(T, pk, m), p);
  return dir == 0 ? 0.5 * (n[1] * phi) : 0.5 * (n[0] * phi);
}
__device__ __noinline__ void tri_dn(const RadialView<double> &T, int pk1, int pk2, const double *n, int dir,
                       const double *q, double &vd, double &vq) {
  double r1sq = 0.0, r2sq = 0.0, dot = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double r1 = q[a] - q[3 + a], r2 = q[a] - q[6 + a];
    r1sq += sqz(r1);
    r2sq += sqz(r2);
    dot += r1 * r2;
  }
  double p1, p2;
  const int m1 = seg_ref(sqrt(r1sq), T.dx, T.n, p1), m2 = seg_ref(sqrt(r2sq), T.dx, T.n, p2);
  double k1[8], k2[8];
  ld8(uw_rec(T, pk1, m1), k1);
  ld8(uw_rec(T, pk2, m2), k2);
  const double s1 = cubv(k1, p1), s2 = cubv(k2, p2);          // u
  const double t1 = cubv(k1 + 4, p1), t2 = cubv(k2 + 4, p2);  // w
  if (dir == 0) {
    const double u1 = n[0] * n[1] * s1, u2 = n[0] * n[2] * s2;
    const double d1 = n[1] * s1, d2 = n[2] * s2;
    vd = (1.0 / 2.0) * d1 * u2 * dot + (1.0 / 2.0) * u1 * d2 * dot;
    const double w1 = n[0] * n[1] * t1, w2 = n[0] * n[2] * t2;
    const double e1 = n[1] * t1, e2 = n[2] * t2, dd = sqz(dot);
    vq = (1.0 / 2.0) * e1 * w2 * dd + (1.0 / 2.0) * w1 * e2 * dd -
         (1.0 / 6.0) * e1 * w2 * r1sq * r2sq - (1.0 / 6.0) * w1 * e2 * r1sq * r2sq;
  } else if (dir == 1) {
    vd = (1.0 / 2.0) * (n[0] * s1) * (n[0] * n[2] * s2) * dot;
    const double e1 = n[0] * t1, w2 = n[0] * n[2] * t2;
    vq = (1.0 / 2.0) * e1 * w2 * sqz(dot) - (1.0 / 6.0) * e1 * w2 * r1sq * r2sq;
  } else {
    vd = (1.0 / 2.0) * (n[0] * n[1] * s1) * (n[0] * s2) * dot;
    const double w1 = n[0] * n[1] * t1, e2 = n[0] * t2;
    vq = (1.0 / 2.0) * w1 * e2 * sqz(dot) - (1.0 / 6.0) * w1 * e2 * r1sq * r2sq;
  }
}

// Degree-3 rule points of a measure (Quadrature-Measure.cpp:30-109,
// Quadrature-Hermitian-3th.cpp:36-110): slots grouped (a coincident j1 = j2
// is one group), one row per axis of each group, 2D points
// mean +/- sqrt(2) sigma_s zeta [slot s in row l's group, axis of row l],
// zeta = sqrt(D) / sqrt(2), weight 1 / (2D).
struct Gh3 {
  int ns, D, grp[3];
};
__device__ __forceinline__ Gh3 gh3_of(int ns, bool coincident) {
  Gh3 m;
  m.ns = ns;
  m.grp[0] = 0;
  m.grp[1] = 1;
  m.grp[2] = coincident ? 1 : 2;
  m.D = 3 * (ns == 2 ? 2 : (coincident ? 2 : 3));
  return m;
}
template <int N>
__device__ __forceinline__ void gh3_point(const Gh3 &m, const double (&mean)[N], const double *sig,
                                          int l, double sgn, double (&ql)[N]) {
  const double zeta = sqrt((double)m.D) / kSqrt2d;
  for (int s = 0; s < m.ns; ++s)
    for (int a = 0; a < 3; ++a) {
      const double b = (m.grp[s] == l / 3 && a == l % 3) ? 1.0 : 0.0;
      const double off = kSqrt2d * sig[s] * zeta * b;
      ql[s * 3 + a] = sgn > 0 ? mean[s * 3 + a] + off : mean[s * 3 + a] - off;
    }
}

// Five-point second difference with step 0.01 (meanfield_integral_mp_dmq).
__device__ __forceinline__ double d2_dmq(double gpp, double gp, double g0, double gm,
                                         double gmm) {
  const double dr = 0.01;
  return (-gpp + 16.0 * gp - 30.0 * g0 + 16.0 * gm - gmm) / (12.0 * dr * dr);
}
template <int N>
__device__ __forceinline__ void moved(const double (&q)[N], int k, int which, double (&o)[N]) {
  const double dr = 0.01;
#pragma unroll
  for (int c = 0; c < N; ++c) o[c] = q[c];
  o[k] = which == 0 ? q[k] + dr * 2 : which == 1 ? q[k] + dr : which == 2 ? q[k] - dr
                                                                            : q[k] - dr * 2;
}

// meanfield_integral_mp_dmq of rho_ij and V_pair_ij over the pair measure
// (c, nb) for slot `dir`: the gradient at the mean plus sigma_s^2 / 2 times
// its five-point second differences in every coordinate of both slots.
__device__ void pair_dmq(const RadialView<double> &T, const PairSite &c, const PairSite &nb,
                         int dir, double *drho, double *dpair) {
  const int pk = pair_kind(c.code, nb.code);
  const double q[6] = {c.q[0], c.q[1], c.q[2], nb.q[0], nb.q[1], nb.q[2]};
  const double sig[2] = {c.sig, nb.sig};
  double g0r[3], g0p[3];
  rho_dq(T, pk, nb.code, nb.x, dir, q, g0r);
  pair_dq(T, pk, c.x, nb.x, dir, q, g0p);
  for (int a = 0; a < 3; ++a) {
    drho[a] = g0r[a];
    dpair[a] = g0p[a];
  }
  for (int s = 0; s < 2; ++s) {
    const double c2 = sqz(sig[s]) / 2.0;
    for (int al = 0; al < 3; ++al) {
      double gr[4][3], gp[4][3];
      for (int w = 0; w < 4; ++w) {
        double qq[6];
        moved(q, 3 * s + al, w, qq);
        rho_dq(T, pk, nb.code, nb.x, dir, qq, gr[w]);
        pair_dq(T, pk, c.x, nb.x, dir, qq, gp[w]);
      }
      for (int b = 0; b < 3; ++b) {
        drho[b] += c2 * d2_dmq(gr[0][b], gr[1][b], g0r[b], gr[2][b], gr[3][b]);
        dpair[b] += c2 * d2_dmq(gp[0][b], gp[1][b], g0p[b], gp[2][b], gp[3][b]);
      }
    }
  }
}

// meanfield_integral_mp_dmq of V_dipole and V_quadrupole over the triplet
// measure (c, j1, j2) for slot `dir`; every slot moves alone.
__device__ void tri_dmq(const RadialView<double> &T, const PairSite &c, const PairSite &j1,
                        const PairSite &j2, int dir, double *gdip, double *gquad) {
  const int pk1 = pair_kind(c.code, j1.code), pk2 = pair_kind(c.code, j2.code);
  const double n[3] = {c.x, j1.x, j2.x};
  const double q[9] = {c.q[0],  c.q[1],  c.q[2],  j1.q[0], j1.q[1],
                       j1.q[2], j2.q[0], j2.q[1], j2.q[2]};
  const double sig[3] = {c.sig, j1.sig, j2.sig};
  double g0d[3], g0q[3];
  tri_dq(T, pk1, pk2, n, dir, q, g0d, g0q);
  for (int a = 0; a < 3; ++a) {
    gdip[a] = g0d[a];
    gquad[a] = g0q[a];
  }
  for (int s = 0; s < 3; ++s) {
    const double c2 = sqz(sig[s]) / 2.0;
    for (int al = 0; al < 3; ++al) {
      double gd[4][3], gq[4][3];
      for (int w = 0; w < 4; ++w) {
        double qq[9];
        moved(q, 3 * s + al, w, qq);
        tri_dq(T, pk1, pk2, n, dir, qq, gd[w], gq[w]);
      }
      for (int b = 0; b < 3; ++b) {
        gdip[b] += c2 * d2_dmq(gd[0][b], gd[1][b], g0d[b], gd[2][b], gd[3][b]);
        gquad[b] += c2 * d2_dmq(gq[0][b], gq[1][b], g0q[b], gq[2][b], gq[3][b]);
      }
    }
  }
}

// One pair measure (c = slot 0, nb = slot 1) for u in slot `dir`: the
// multipole dmq and dsq of rho and of the pair term, and the degree-3 dxi.
struct PairOut {
  double drho_q[3], pair_q[3], drho_s, pair_s, drho_x, pair_x;
};
__device__ __noinline__ void pair_residual(const RadialView<double> &T, int rule, const PairSite &c,
                              const PairSite &nb, int dir, PairOut &o) {
  const int pk = pair_kind(c.code, nb.code);
  const double q[6] = {c.q[0], c.q[1], c.q[2], nb.q[0], nb.q[1], nb.q[2]};
  const double sig[2] = {c.sig, nb.sig}, n[2] = {c.x, nb.x};
  pair_dmq(T, c, nb, dir, o.drho_q, o.pair_q);
  // dsq: sigma_dir x tr of block (dir, dir)
  o.drho_s = 0.0;
  o.pair_s = 0.0;
  if (rule == 1) {
    const double f0r = rho_F_call(T, pk, nb.code, nb.x, q), f0p = pair_F_call(T, pk, c.x, nb.x, q);
    for (int al = 0; al < 3; ++al) {
      double fr[4], fp[4];
      for (int w = 0; w < 4; ++w) {
        double qq[6];
        shifted(q, 3 * dir + al, w, qq);
        fr[w] = rho_F_call(T, pk, nb.code, nb.x, qq);
        fp[w] = pair_F_call(T, pk, c.x, nb.x, qq);
      }
      o.drho_s += sig[dir] * d2_5(fr[0], fr[1], f0r, fr[2], fr[3]);
      o.pair_s += sig[dir] * d2_5(fp[0], fp[1], f0p, fp[2], fp[3]);
    }
  } else {
    double r2 = 0.0;
    for (int a = 0; a < 3; ++a) r2 += sqz(q[a] - q[3 + a]);
    const double s = sqrt(r2);
    double p;
    const int m = seg_ref(s, T.dx, T.n, p);
    const double *kr = pr_rec(T, pk, m) + rho_off(pk, nb.code), *kp = pr_rec(T, pk, m);
    o.drho_s = sig[dir] * (nb.x * (cubdd(kr, p) + 2.0 * cubd(kr, p) / s));
    o.pair_s = sig[dir] * (0.5 * c.x * nb.x * (cubdd(kp, p) + 2.0 * cubd(kp, p) / s));
  }
  // dxi on the degree-3 rule
  const Gh3 g = gh3_of(2, false);
  const double W = 1.0 / (2.0 * g.D);
  o.drho_x = 0.0;
  o.pair_x = 0.0;
  for (int sg = 0; sg < 2; ++sg)
    for (int l = 0; l < g.D; ++l) {
      double ql[6];
      gh3_point(g, q, sig, l, sg == 0 ? 1.0 : -1.0, ql);
      o.drho_x += rho_dn(T, pk, nb.code, dir, ql) * W;
      o.pair_x += pair_dn(T, pk, n, dir, ql) * W;
    }
}

// ---- triplets: every slot direction from one set of leg evaluations ------
// One leg (i, j_k) of a triplet geometry: r = q_i - q_jk, |r|^2, |r|, 1/|r|
// and the raw spline values (D: and first derivatives) of u and w at |r|,
// each formed in the operations of tri_F, tri_dq and tri_dn, so a term
// assembled from legs equals theirs bit for bit.  A finite-difference or
// rule point that moves one slot recomputes only the legs that slot ends.
struct Leg {
  double r[3], rsq, nr, inv, u, du, w, dw;
};
template <bool D>
__device__ __forceinline__ void leg_of(const RadialView<double> &T, int pk, const double *qi,
                                       const double *qj, Leg &L) {
  L.rsq = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    L.r[a] = qi[a] - qj[a];
    L.rsq += sqz(L.r[a]);
  }
  L.nr = sqrt(L.rsq);
  double p;
  const int m = seg_ref(L.nr, T.dx, T.n, p);
  double k[8];
  ld8(uw_rec(T, pk, m), k);
  L.u = cubv(k, p);
  L.w = cubv(k + 4, p);
  if (D) {
    L.inv = 1.0 / L.nr;
    L.du = cubd(k, p);
    L.dw = cubd(k + 4, p);
  }
}
// A leg parked in shared memory (10 doubles) while other work holds the
// registers.
__device__ __forceinline__ void st_leg(double *p, const Leg &L) {
  p[0] = L.r[0]; p[1] = L.r[1]; p[2] = L.r[2]; p[3] = L.rsq; p[4] = L.nr;
  p[5] = L.inv; p[6] = L.u; p[7] = L.du; p[8] = L.w; p[9] = L.dw;
}
__device__ __forceinline__ Leg ld_leg(const double *p) {
  Leg L;
  L.r[0] = p[0]; L.r[1] = p[1]; L.r[2] = p[2]; L.rsq = p[3]; L.nr = p[4];
  L.inv = p[5]; L.u = p[6]; L.du = p[7]; L.w = p[8]; L.dw = p[9];
  return L;
}
__device__ __forceinline__ double leg_dot(const Leg &L1, const Leg &L2) {
  double dot = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) dot += L1.r[a] * L2.r[a];
  return dot;
}
// tri_dq of all three slots, component e = 6 dir + a (dipole) or
// 6 dir + 3 + a (quadrupole), each handed to sink(e, value) as it is formed.
template <class Sink>
__device__ __forceinline__ void dq_all(const Leg &L1, const Leg &L2, double c1, double c2,
                                       Sink &&sink) {
  const double dot = leg_dot(L1, L2);
  const double i1 = L1.inv, i2 = L2.inv, n1 = L1.nr, n2 = L2.nr;
  const double r1sq = L1.rsq, r2sq = L2.rsq;
  const double u1 = c1 * L1.u, u2 = c2 * L2.u;
  const double du1 = c1 * L1.du, du2 = c2 * L2.du;
  const double w1 = c1 * L1.w, w2 = c2 * L2.w;
  const double dw1 = c1 * L1.dw, dw2 = c2 * L2.dw;
  const double dd = sqz(dot);
  const double *r1 = L1.r, *r2 = L2.r;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    sink(a, 0.5 * (du1 * u2 * dot * i1 * r1[a] + u1 * du2 * dot * i2 * r2[a] +
                   u1 * u2 * (r1[a] + r2[a])));
    sink(3 + a, (1.0 / 2.0) * (dw1 * w2 * dd * i1 * r1[a] + w1 * dw2 * dd * i2 * r2[a] +
                               w1 * w2 * 2 * dot * (r1[a] + r2[a])) -
                    (1.0 / 6.0) * (dw1 * w2 * n1 * r2sq * r1[a] + w1 * dw2 * r1sq * n2 * r2[a] +
                                   w1 * w2 * 2 * r2sq * r1[a] + w1 * w2 * 2 * r1sq * r2[a]));
    sink(6 + a, -0.5 * (du1 * u2 * dot * i1 * r1[a] + u1 * u2 * r2[a]));
    sink(9 + a, -0.5 * (dw1 * w2 * dd * i1 * r1[a] + w1 * w2 * 2 * dot * r2[a]) +
                    (1.0 / 6.0) * (dw1 * w2 * n1 * r2sq * r1[a] + w1 * w2 * 2 * r2sq * r1[a]));
    sink(12 + a, -0.5 * (u1 * du2 * dot * i2 * r2[a] + u1 * u2 * r1[a]));
    sink(15 + a, -0.5 * (w1 * dw2 * dd * i2 * r2[a] + w1 * w2 * 2 * dot * r1[a]) +
                     (1.0 / 6.0) * (w1 * dw2 * r1sq * n2 * r2[a] + w1 * w2 * 2 * r1sq * r2[a]));
  }
}
// tri_F from legs.
__device__ __forceinline__ void f_legs(const Leg &L1, const Leg &L2, double c1, double c2,
                                       double &fd, double &fq) {
  const double dot = leg_dot(L1, L2);
  const double u1 = c1 * L1.u, u2 = c2 * L2.u;
  const double w1 = c1 * L1.w, w2 = c2 * L2.w;
  fd = (1.0 / 2.0) * u1 * u2 * dot;
  fq = (1.0 / 2.0) * w1 * w2 * sqz(dot) - (1.0 / 6.0) * w1 * w2 * L1.rsq * L2.rsq;
}
// tri_dn of all three slots: v[2 dir] dipole, v[2 dir + 1] quadrupole.
__device__ __forceinline__ void dn_all(const Leg &L1, const Leg &L2, const double *n,
                                       double (&v)[6]) {
  const double dot = leg_dot(L1, L2);
  const double r1sq = L1.rsq, r2sq = L2.rsq;
  const double s1 = L1.u, s2 = L2.u, t1 = L1.w, t2 = L2.w;
  {
    const double u1 = n[0] * n[1] * s1, u2 = n[0] * n[2] * s2;
    const double d1 = n[1] * s1, d2 = n[2] * s2;
    v[0] = (1.0 / 2.0) * d1 * u2 * dot + (1.0 / 2.0) * u1 * d2 * dot;
    const double w1 = n[0] * n[1] * t1, w2 = n[0] * n[2] * t2;
    const double e1 = n[1] * t1, e2 = n[2] * t2, dd = sqz(dot);
    v[1] = (1.0 / 2.0) * e1 * w2 * dd + (1.0 / 2.0) * w1 * e2 * dd -
           (1.0 / 6.0) * e1 * w2 * r1sq * r2sq - (1.0 / 6.0) * w1 * e2 * r1sq * r2sq;
  }
  {
    v[2] = (1.0 / 2.0) * (n[0] * s1) * (n[0] * n[2] * s2) * dot;
    const double e1 = n[0] * t1, w2 = n[0] * n[2] * t2;
    v[3] = (1.0 / 2.0) * e1 * w2 * sqz(dot) - (1.0 / 6.0) * e1 * w2 * r1sq * r2sq;
  }
  {
    v[4] = (1.0 / 2.0) * (n[0] * n[1] * s1) * (n[0] * s2) * dot;
    const double w1 = n[0] * n[1] * t1, e2 = n[0] * t2;
    v[5] = (1.0 / 2.0) * w1 * e2 * sqz(dot) - (1.0 / 6.0) * w1 * e2 * r1sq * r2sq;
  }
}

// dmq of every slot's three coordinates: for each, the five-point second
// difference (step 0.01) of all slots' gradients, times sigma_S^2 / 2, added
// to acc (g0: the gradients at the mean).  g0, acc and the legs at the mean
// are the lane's shared-memory scratch.  One body serves the three slots (a
// moved slot recomputes the legs it ends, the others come from the
// scratch), which keeps the unrolled differences small enough for the
// instruction cache.
__device__ __forceinline__ void dmq_slots(const RadialView<double> &T, int pk1, int pk2,
                                          const double (&q)[9], const double (&sig)[3],
                                          const double *legs, double c1, double c2,
                                          const double *g0, double *acc) {
#pragma unroll 1
  for (int S = 0; S < 3; ++S) {
    const double c2s = sqz(S == 0 ? sig[0] : S == 1 ? sig[1] : sig[2]) / 2.0;
    double base[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) base[a] = S == 0 ? q[a] : S == 1 ? q[3 + a] : q[6 + a];
#pragma unroll 1
    for (int al = 0; al < 3; ++al) {
      const double dr = 0.01;
      const double x0 = al == 0 ? base[0] : al == 1 ? base[1] : base[2];
      double t[18];
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        const double v = w == 0 ? x0 + dr * 2 : w == 1 ? x0 + dr : w == 2 ? x0 - dr
                                                                          : x0 - dr * 2;
        double pc[3], p1[3], p2[3];  // the three positions with slot S moved
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double m = a == al ? v : base[a];
          pc[a] = S == 0 ? m : q[a];
          p1[a] = S == 1 ? m : q[3 + a];
          p2[a] = S == 2 ? m : q[6 + a];
        }
        // the five-point combination -gpp + 16 gp - 30 g0 + 16 gm - gmm,
        // formed in that order as the points arrive (pp, p, m, mm)
        auto step = [&](int e, double g) {
          if (w == 0) t[e] = -g;
          else if (w == 1) t[e] = (t[e] + 16.0 * g) - 30.0 * g0[e];
          else if (w == 2) t[e] = t[e] + 16.0 * g;
          else t[e] = t[e] - g;
        };
        Leg M1, M2;
        if (S != 2) leg_of<true>(T, pk1, pc, p1, M1);
        else M1 = ld_leg(legs);
        if (S != 1) leg_of<true>(T, pk2, pc, p2, M2);
        else M2 = ld_leg(legs + 10);
        dq_all(M1, M2, c1, c2, step);
      }
#pragma unroll
      for (int e = 0; e < 18; ++e) acc[e] += c2s * (t[e] / (12.0 * dr * dr));
    }
  }
}

// Second differences (step 1e-4) of the dipole and quadrupole values along
// slot S's three coordinates (the reference's d2F_dq2_FD diagonal).
template <int S>
__device__ __forceinline__ void fd_slot(const RadialView<double> &T, int pk1, int pk2,
                                        const double (&q)[9], const double *legs,
                                        double c1, double c2, double f0d, double f0q,
                                        double *dd, double *dq) {
#pragma unroll 1
  for (int al = 0; al < 3; ++al) {
    const double dr = 0.0001;
    const double x0 = al == 0 ? q[3 * S] : al == 1 ? q[3 * S + 1] : q[3 * S + 2];
    double fd4[4], fq4[4];
#pragma unroll 1
    for (int w = 0; w < 4; ++w) {
      const double D = 1.0;
      const double v = w == 0 ? x0 + D * dr * 2 : w == 1 ? x0 + D * dr
                     : w == 2 ? x0 - D * dr : x0 - D * dr * 2;
      double pm[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) pm[a] = a == al ? v : q[3 * S + a];
      double fd, fq;
      if (S == 0) {
        Leg M1, M2;
        leg_of<false>(T, pk1, pm, q + 3, M1);
        leg_of<false>(T, pk2, pm, q + 6, M2);
        f_legs(M1, M2, c1, c2, fd, fq);
      } else if (S == 1) {
        Leg M1;
        leg_of<false>(T, pk1, q, pm, M1);
        f_legs(M1, ld_leg(legs + 10), c1, c2, fd, fq);
      } else {
        Leg M2;
        leg_of<false>(T, pk2, q, pm, M2);
        f_legs(ld_leg(legs), M2, c1, c2, fd, fq);
      }
      if (w == 0) { fd4[0] = fd; fq4[0] = fq; }
      else if (w == 1) { fd4[1] = fd; fq4[1] = fq; }
      else if (w == 2) { fd4[2] = fd; fq4[2] = fq; }
      else { fd4[3] = fd; fq4[3] = fq; }
    }
    const double vd = d2_5(fd4[0], fd4[1], f0d, fd4[2], fd4[3]);
    const double vq = d2_5(fq4[0], fq4[1], f0q, fq4[2], fq4[3]);
    if (al == 0) { dd[0] = vd; dq[0] = vq; }
    else if (al == 1) { dd[1] = vd; dq[1] = vq; }
    else { dd[2] = vd; dq[2] = vq; }
  }
}

// One triplet measure (c; j1, j2) for u in each slot (dir 0: c, 1: j1,
// 2: j2; with j1 = j2 the coincident measure), evaluate_DV0_i_Dq_u_MgHx's
// meanfield_integral_mp_dmq and _dsq of the dipole and quadrupole terms
// (with_q: j2 passes the gradient's x > min_occupancy test) and
// evaluate_DV0_i_Dxi_u_adp_MgHx's degree-3 dxi (j2 passes x >=
// min_occupancy, as every triplet here does).  Each slot's values are the
// reference's, term for term: the same points, the same differences, the
// same per-slot sums; only the geometry is shared between the slots.
// out[5 dir + 0..2] = dmq dipole + quadrupole, [3] dsq, [4] dxi, times f
// (the lane's shared-memory stage); sc: 56 doubles of its scratch.
__device__ __forceinline__ void tri_all(const RadialView<double> &T, int rule, const PairSite &c,
                                        const PairSite &j1, const PairSite &j2,
                                        bool coincident, bool with_q, double f, double *sc,
                                        double *out) {
  const int pk1 = pair_kind(c.code, j1.code), pk2 = pair_kind(c.code, j2.code);
  const double n[3] = {c.x, j1.x, j2.x};
  const double c1 = n[0] * n[1], c2 = n[0] * n[2];
  const double q[9] = {c.q[0],  c.q[1],  c.q[2],  j1.q[0], j1.q[1],
                       j1.q[2], j2.q[0], j2.q[1], j2.q[2]};
  const double sig[3] = {c.sig, j1.sig, j2.sig};
  // the legs at the mean, parked in the scratch (sc[36..55])
  double *legs = sc + 36;
  {
    Leg L1, L2;
    leg_of<true>(T, pk1, q, q + 3, L1);
    leg_of<true>(T, pk2, q, q + 6, L2);
    st_leg(legs, L1);
    st_leg(legs + 10, L2);
  }
#pragma unroll
  for (int e = 0; e < 15; ++e) out[e] = 0.0;
  if (with_q) {
    // dmq: the gradients at the mean plus sigma_s^2 / 2 times their
    // second differences along every coordinate of every slot
    double *g0 = sc, *acc = sc + 18;
    dq_all(ld_leg(legs), ld_leg(legs + 10), c1, c2,
           [&](int e, double g) { g0[e] = acc[e] = g; });
    dmq_slots(T, pk1, pk2, q, sig, legs, c1, c2, g0, acc);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int a = 0; a < 3; ++a) out[5 * d + a] = f * acc[6 * d + a] + f * acc[6 * d + 3 + a];
    // dsq: sigma_dir x the block traces of the dof row of dir
    double sd_[3] = {0, 0, 0}, sq_[3] = {0, 0, 0};
    if (rule == 1) {
      double f0d, f0q;
      f_legs(ld_leg(legs), ld_leg(legs + 10), c1, c2, f0d, f0q);
      // the second differences in the scratch: Dd[slot][al] at sc[3 slot +
      // al], Dq at sc[9 + 3 slot + al]
      double *Dd = sc, *Dq = sc + 9;
      fd_slot<0>(T, pk1, pk2, q, legs, c1, c2, f0d, f0q, Dd, Dq);
      fd_slot<1>(T, pk1, pk2, q, legs, c1, c2, f0d, f0q, Dd + 3, Dq + 3);
      fd_slot<2>(T, pk1, pk2, q, legs, c1, c2, f0d, f0q, Dd + 6, Dq + 6);
      // rows of the dof table in the reference's (dir, b) order; direction
      // dir * 3 + b reads slot (dir * 3 + b) / 4
#pragma unroll
      for (int dir = 0; dir < 3; ++dir)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          if (!(b == dir || (coincident && dir > 0 && b > 0))) continue;
          const int dirn = dir * 3 + b, slot = dirn / 4;
          const bool diag = dirn == 0 || dirn == 4 || dirn == 8;
#pragma unroll
          for (int al = 0; al < 3; ++al) {
            sd_[dir] += sig[dir] * Dd[3 * slot + al];
            if (diag) sq_[dir] += sig[dir] * Dq[3 * slot + al];
          }
        }
    } else {
      const TriTr t = tri_traces_call(T, pk1, pk2, n, q);
#pragma unroll
      for (int dir = 0; dir < 3; ++dir)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          if (!(b == dir || (coincident && dir > 0 && b > 0))) continue;
          double trd, trq;
          if (b != dir) {
            trd = t.d12;
            trq = t.q12;
          } else if (dir == 0) {
            trd = t.d11 + t.d22 + 2.0 * t.d12;
            trq = t.q11 + t.q22 + 2.0 * t.q12;
          } else {
            trd = dir == 1 ? t.d11 : t.d22;
            trq = dir == 1 ? t.q11 : t.q22;
          }
          sd_[dir] += sig[dir] * trd;
          sq_[dir] += sig[dir] * trq;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) out[5 * d + 3] = f * sd_[d] + f * sq_[d];
  }
  // dxi on the degree-3 rule: the rows of a group move the group's slots
  const Gh3 g = gh3_of(3, coincident);
  const double W = 1.0 / (2.0 * g.D);
  double vx[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
  for (int sg = 0; sg < 2; ++sg)
#pragma unroll 1
    for (int l = 0; l < g.D; ++l) {
      double ql[9];
      gh3_point(g, q, sig, l, sg == 0 ? 1.0 : -1.0, ql);
      const int grp = l / 3;
      Leg M1, M2;
      if (grp == 0 || grp == g.grp[1]) leg_of<false>(T, pk1, ql, ql + 3, M1);
      else M1 = ld_leg(legs);
      if (grp == 0 || grp == g.grp[2]) leg_of<false>(T, pk2, ql, ql + 6, M2);
      else M2 = ld_leg(legs + 10);
      double v[6];
      dn_all(M1, M2, n, v);
#pragma unroll
      for (int e = 0; e < 6; ++e) vx[e] += v[e] * W;
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) out[5 * d + 4] = f * vx[2 * d] + f * vx[2 * d + 1];
}

struct MpResArgs {
  MpArgs b;
  const int *owner;
  const int *rev;      // reverse slot of every real list entry (-1: none)
  const double *gamma;
  double *gk;  // 5 values per (centre o, slot): slot 0 the pair (o, o), 1 + k list entry k
  double *g5;  // the same per (u, centre): centre 0 u itself, 1 + k u's list entry k
  double *Rq, *Rs, *Rx;
};

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// One warp per centre o: every term of evaluate_DV0_i_Dq_u_MgHx and
// evaluate_DV0_i_Dxi_u_adp_MgHx (i = o) for u = o and for u = each entry of
// o's list, the pairs (o, j) and the triplets (o; j1 <= j2) of o's active
// entries (x >= min_occupancy; an empty site takes part in nothing), one
// pair or triplet per lane.  A triplet gives its slots' values to u = o
// (slot 0), u = j1 (slot 1) and u = j2 (slot 2) at once.  The per-(o, u)
// totals gather in shared memory in a fixed order (the lanes stage their
// values, then one lane per value adds them in lane order), so every
// evaluation gives the same bits.
constexpr int kMpW = 1;              // warps per block
constexpr int kMpSlots = 256;        // maxneigh + 1
__global__ void __launch_bounds__(kMpW * 32) mp_centre_kernel(MpResArgs r) {
  const MpArgs &a = r.b;
  __shared__ double acc_s[kMpW][kMpSlots][5];
  __shared__ double stage_s[kMpW][32][15];  // per lane: its triplet's 15 values
  __shared__ int key_s[kMpW][32][2];
  __shared__ int act_s[kMpW][kMpSlots];
  __shared__ double scr_s[kMpW][32][57];  // tri_all's per-lane scratch (odd stride)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int o = blockIdx.x * kMpW + warp;
  if (o >= a.n_real) return;
  double(*acc)[5] = acc_s[warp];
  int *act = act_s[warp];
  const int nb0 = a.offs[o], nn = a.offs[o + 1] - nb0;
  if (nn >= kMpSlots) {  // longer than maxneigh lists are refused when built
    for (int e = lane; e < 5 * (1 + nn); e += 32) r.gk[5 * ((size_t)nb0 + o) + e] = nan("");
    return;
  }
  for (int k = lane; k < 1 + nn; k += 32)
    for (int c = 0; c < 5; ++c) acc[k][c] = 0.0;
  const PairSite so = site_of(a, o);
  const bool live = !(so.x < kMinOcc);
  // active entries in list order
  int na = 0;
  for (int base = 0; base < nn; base += 32) {
    const int k = base + lane;
    const bool on = live && k < nn && !(a.xb[a.idx[nb0 + k]].x < kMinOcc);
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (on) act[na + __popc(m & ((1u << lane) - 1u))] = k;
    na += __popc(m);
  }
  __syncwarp();
  double dF = 0.0, Fv = 0.0;
  if (live) {
    double p;
    const SplineView<double> &E = so.code == 0 ? a.emb_mg : a.emb_h;
    const int m = seg_ref(a.rho[o], E.dx, E.n, p);
    const Coef4<double> cf = E.c[m];
    const double kk4[4] = {cf.a, cf.b, cf.c, cf.d};
    dF = cubd(kk4, p);
    Fv = cubv(kk4, p);
  }
  const double fx = so.x * dF;  // the embedding factor of the rho terms
  // pairs: slot 0 (u = o) summed over lanes, slot 1 + k (u = entry k) once
  double ps[5] = {0, 0, 0, 0, 0};
  for (int m = lane; m < na; m += 32) {
    const int k = act[m];
    const PairSite sj = site_of(a, a.idx[nb0 + k]);
    PairOut p0, p1;
    pair_residual(a.T, a.rule, so, sj, 0, p0);
    pair_residual(a.T, a.rule, so, sj, 1, p1);
    for (int b = 0; b < 3; ++b) ps[b] += fx * p0.drho_q[b] + p0.pair_q[b];
    ps[3] += fx * p0.drho_s + p0.pair_s;
    ps[4] += (so.code == 0 ? dF * p0.drho_x : 0.0) + p0.pair_x;
    for (int b = 0; b < 3; ++b) acc[1 + k][b] = fx * p1.drho_q[b] + p1.pair_q[b];
    acc[1 + k][3] = fx * p1.drho_s + p1.pair_s;
    acc[1 + k][4] = (so.code == 1 ? so.x * dF : dF) * p1.drho_x + p1.pair_x;
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) ps[c] = warp_sum(ps[c]);
  __syncwarp();
  if (lane == 0) {
    for (int c = 0; c < 5; ++c) acc[0][c] = ps[c];
    if (live && so.code == 1) acc[0][4] += Fv;  // d(x_o F(rho_o))/dx_o's F part
  }
  __syncwarp();
  // triplets (m1 <= m2) of the active entries, 32 per round
  const long long ntri = (long long)na * (na + 1) / 2;
  for (long long t0 = 0; t0 < ntri; t0 += 32) {
    const long long t = t0 + lane;
    int k1 = -1, k2 = -1;
    double *out = stage_s[warp][lane];
    if (t < ntri) {
      int m2 = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
      while ((long long)m2 * (m2 + 1) / 2 > t) --m2;
      while ((long long)(m2 + 1) * (m2 + 2) / 2 <= t) ++m2;
      const int m1 = (int)(t - (long long)m2 * (m2 + 1) / 2);
      k1 = act[m1];
      k2 = act[m2];
      const PairSite s1 = site_of(a, a.idx[nb0 + k1]);
      const PairSite s2 = site_of(a, a.idx[nb0 + k2]);
      tri_all(a.T, a.rule, so, s1, s2, m1 == m2, !(s2.x <= kMinOcc), m1 == m2 ? 1.0 : 2.0,
              scr_s[warp][lane], out);
    }
    key_s[warp][lane][0] = k1;
    key_s[warp][lane][1] = k2;
    __syncwarp();
    if (lane < 5) {
      for (int l = 0; l < 32; ++l) {
        const int q1 = key_s[warp][l][0], q2 = key_s[warp][l][1];
        if (q1 < 0) break;
        acc[0][lane] += stage_s[warp][l][lane];
        acc[1 + q1][lane] += stage_s[warp][l][5 + lane];
        acc[1 + q2][lane] += stage_s[warp][l][10 + lane];
      }
    }
    __syncwarp();
  }
  double *g = r.gk + 5 * ((size_t)nb0 + o);
  for (int e = lane; e < 5 * (1 + nn); e += 32) g[e] = (&acc[0][0])[e];
}

// The per-(u, centre) layout of the pairs' values: centre 0 is u's own slot
// 0; centre 1 + k (list entry p = offs[u] + k, owner o) is the slot of o's
// entry that is u, seen from o (the reverse slot of p).
__global__ void __launch_bounds__(128) mp_gather_kernel(MpResArgs r) {
  const MpArgs &a = r.b;
  const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= a.n_real) return;
  const int nb0 = a.offs[u], nn = a.offs[u + 1] - nb0;
  double *dst = r.g5 + 5 * ((size_t)nb0 + u);
  for (int c = lane; c < 1 + nn; c += 32) {
    const double *src = nullptr;
    if (c == 0) {
      src = r.gk + 5 * ((size_t)nb0 + u);
    } else {
      const int p = nb0 + c - 1, rv = r.rev[p];
      if (rv >= 0) src = r.gk + 5 * ((size_t)rv + r.owner[a.idx[p]] + 1);
    }
    for (int e = 0; e < 5; ++e) dst[5 * c + e] = src ? src[e] : 0.0;
  }
}

// Residual assembly per real site (the project's definition, include/btam.h):
// R = sum over the centres of beta_o / beta_u times the per-pair values,
// then the entropy and chemical-potential parts.
__global__ void mp_assemble_kernel(MpResArgs r) {
  const MpArgs &a = r.b;
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.n_real) return;
  double rq[3] = {0, 0, 0}, rs = 0.0, rx = 0.0;
  const double2 xbu = a.xb[u];
  const double xu = xbu.x, bu = xbu.y;
  if (!(xu < kMinOcc)) {
    const long long base = (long long)a.offs[u] + u;
    const int ncen = 1 + a.offs[u + 1] - a.offs[u];
    for (int c = 0; c < ncen; ++c) {
      const int ic = c == 0 ? u : a.idx[a.offs[u] + c - 1];
      const int o = r.owner[ic];
      const double wgt = a.xb[o].y / bu;
      const double *g = r.g5 + 5 * (base + c);
      for (int b = 0; b < 3; ++b) rq[b] += wgt * g[b];
      rs += wgt * g[3];
      rx += wgt * g[4];
    }
    rs -= 3.0 / (bu * a.pos[u].w);
    if (a.code[u] == 1) {
      const double dlogz = 3.0 / (2.0 * xu) + (xu < 1.0 ? 1.0 / (1.0 - xu) : 0.0);
      rx -= dlogz / bu;
      if (xu < 0.9999) rx -= r.gamma[u] / bu;
    } else {
      rx = 0.0;
    }
  }
  for (int b = 0; b < 3; ++b) r.Rq[3 * (size_t)u + b] = rq[b];
  r.Rs[u] = rs;
  r.Rx[u] = rx;
}

// evaluate_DV0_i_dF_bulk_MgHx (MgHx-mf-V-bulk.cpp:2329-2552) under the rule,
// at reference positions q0 = q: for every term of V0_i, each slot a's
// meanfield_integral_mp_dmq (x) q_a, summed; W0_i = x_i F'(rho_i) drho +
// pair + dipole + quadrupole (3x3, row: gradient component).  j1 and j2
// skip empty H sites (2408-2410, 2465-2467).  A warp per real site.
__global__ void __launch_bounds__(128) mp_stress_kernel(MpArgs a, double *W) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.n_real) return;
  const PairSite si = site_of(a, i);
  double drho[9], pair[9], dip[9], quad[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) drho[c] = pair[c] = dip[c] = quad[c] = 0.0;
  const int nb0 = a.offs[i], nn = a.offs[i + 1] - nb0;
  if (!(si.x < kMinOcc)) {
    for (int k = lane; k < nn; k += 32) {
      const PairSite sj = site_of(a, a.idx[nb0 + k]);
      if (empty_h(sj)) continue;
      for (int dir = 0; dir < 2; ++dir) {
        const double *r0 = dir == 0 ? si.q : sj.q;
        double gr[3], gp[3];
        pair_dmq(a.T, si, sj, dir, gr, gp);
        for (int x = 0; x < 3; ++x)
          for (int y = 0; y < 3; ++y) {
            drho[3 * x + y] += gr[x] * r0[y];
            pair[3 * x + y] += gp[x] * r0[y];
          }
      }
    }
    const long long ntri = (long long)nn * (nn + 1) / 2;
    for (long long t = lane; t < ntri; t += 32) {
      int k2 = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
      while ((long long)k2 * (k2 + 1) / 2 > t) --k2;
      while ((long long)(k2 + 1) * (k2 + 2) / 2 <= t) ++k2;
      const int k1 = (int)(t - (long long)k2 * (k2 + 1) / 2);
      const PairSite s1 = site_of(a, a.idx[nb0 + k1]);
      if (empty_h(s1)) continue;
      const PairSite s2 = site_of(a, a.idx[nb0 + k2]);
      if (empty_h(s2)) continue;
      const double f = k1 == k2 ? 1.0 : 2.0;
      for (int dir = 0; dir < 3; ++dir) {
        const double *r0 = dir == 0 ? si.q : (dir == 1 ? s1.q : s2.q);
        double gd[3], gq[3];
        tri_dmq(a.T, si, s1, s2, dir, gd, gq);
        for (int x = 0; x < 3; ++x)
          for (int y = 0; y < 3; ++y) {
            dip[3 * x + y] += f * gd[x] * r0[y];
            quad[3 * x + y] += f * gq[x] * r0[y];
          }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    drho[c] = warp_sum(drho[c]);
    pair[c] = warp_sum(pair[c]);
    dip[c] = warp_sum(dip[c]);
    quad[c] = warp_sum(quad[c]);
  }
  if (lane == 0) {
    double dF = 0.0;
    if (!(si.x < kMinOcc)) {
      const SplineView<double> &E = si.code == 0 ? a.emb_mg : a.emb_h;
      double p;
      const int m = seg_ref(a.rho[i], E.dx, E.n, p);
      const Coef4<double> cf = E.c[m];
      const double k4[4] = {cf.a, cf.b, cf.c, cf.d};
      dF = cubd(k4, p);
    }
    for (int c = 0; c < 9; ++c)
      W[9 * (size_t)i + c] =
          si.x < kMinOcc ? 0.0 : si.x * dF * drho[c] + pair[c] + dip[c] + quad[c];
  }
}

// Per list entry p of a real site i: the multipole rule's gradient of rho_ij
// (j = idx[p]) in q_i (meanfield_integral_mp_dmq), the piece of
// evaluate_D2V0_i_Dmeanq2_u_MgHx the rule changes (MgHx-mf-V-bulk.cpp:1476;
// its blocks stay on meanfield_integral_gh_3th_d2mq, 1482-1566).
__global__ void __launch_bounds__(128) mp_rho_grad_kernel(MpArgs a, double *G) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.n_real) return;
  const PairSite si = site_of(a, i);
  for (int k = a.offs[i] + lane; k < a.offs[i + 1]; k += 32) {
    const PairSite sj = site_of(a, a.idx[k]);
    double gr[3], gp[3];
    pair_dmq(a.T, si, sj, 0, gr, gp);
    for (int c = 0; c < 3; ++c) G[3 * (size_t)k + c] = gr[c];
  }
}

// ---- the per-term plugin interface ------------------------------------------
// The reference's potential_function table (Macros.hpp:252-278) of its four
// ADP terms, rho_ij (MgHx-ADP.cpp:526-844), V_pair_ij (869-1209),
// V_dipole_ij1j2 (1233-1758) and V_quadrupole_ij1j2 (1781-2434), one
// geometry per thread: F, dF_dq, d2F_dq2, dF_dq_FD, d2F_dq2_FD and dF_dn,
// and their averages over the reference's measure with the degree-3 rule.
// Values, gradients, occupancy derivatives and the finite differences use
// the restated functions above (the reference's operation order, no
// contraction); the analytic Hessian blocks are formed here from the
// terms' radial, vector and tensor parts.
struct TermArgs {
  RadialView<double> T;
  int term, fn, dir, ns, n;
  int mode, coincident;   // quadratures
  const double *q, *x, *sigma;
  const int *code;        // 3 per geometry: 0 Mg, 1 H
  double *out;            // 9 per geometry
};

__device__ double term_F(const RadialView<double> &T, int term, const int *c, const double *n,
                         const double (&q)[9]) {
  const int pk1 = pair_kind(c[0], c[1]);
  if (term == 0) return rho_F(T, pk1, c[1], n[1], q);
  if (term == 1) return pair_F(T, pk1, n[0], n[1], q);
  double fd, fq;
  tri_F(T, pk1, pair_kind(c[0], c[2]), n, q, fd, fq);
  return term == 2 ? fd : fq;
}
__device__ void term_dq(const RadialView<double> &T, int term, const int *c, const double *n,
                        int dir, const double *q, double *g) {
  const int pk1 = pair_kind(c[0], c[1]);
  if (term == 0) {
    rho_dq(T, pk1, c[1], n[1], dir, q, g);
  } else if (term == 1) {
    pair_dq(T, pk1, n[0], n[1], dir, q, g);
  } else {
    double gd[3], gq[3];
    tri_dq(T, pk1, pair_kind(c[0], c[2]), n, dir, q, gd, gq);
    for (int a = 0; a < 3; ++a) g[a] = term == 2 ? gd[a] : gq[a];
  }
}
__device__ double term_dn(const RadialView<double> &T, int term, const int *c, const double *n,
                          int dir, const double *q) {
  const int pk1 = pair_kind(c[0], c[1]);
  if (term == 0) return rho_dn(T, pk1, c[1], dir, q);
  if (term == 1) return pair_dn(T, pk1, n, dir, q);
  double vd, vq;
  tri_dn(T, pk1, pair_kind(c[0], c[2]), n, dir, q, vd, vq);
  return term == 2 ? vd : vq;
}

// Spline value and first and second derivatives of four coefficients.
__device__ __forceinline__ void cub3(const double *k, double p, double (&f)[3]) {
  f[0] = cubv(k, p);
  f[1] = cubd(k, p);
  f[2] = cubdd(k, p);
}
// H (3x3) += c (f'' P + f' (I - P) / s), P = r r^T / s^2: the Hessian of
// c f(|r|) in r.
__device__ void hess_radial(const double *r, double s, double d1, double d2, double c,
                            double *H) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double P = r[a] * r[b] / (s * s);
      H[3 * a + b] += c * (d2 * P + d1 * ((a == b ? 1.0 : 0.0) - P) / s);
    }
}

// The analytic Hessian block `dir` of a term at one geometry, as the
// reference's d2F_dq2 numbers them: pairs 0 (i i), 1 and 2 (i j, j i), 3
// (j j); triplets 3 a + b for slots (a, b), of which the reference forms 0,
// 4, 5, 7 and 8 and leaves the others zero.  With r_k = q_0 - q_k, the
// blocks follow from H11 = d2V/dr1^2, H22 and H12 = d2V/dr1 dr2:
// (0, 0) = H11 + H22 + H12 + H12^T, (1, 1) = H11, (2, 2) = H22,
// (1, 2) = H12, (2, 1) = H12^T.
__device__ void term_d2(const RadialView<double> &T, int term, const int *c, const double *n,
                        int dir, const double *q, double *out) {
  for (int e = 0; e < 9; ++e) out[e] = 0.0;
  if (term < 2) {
    const int pk = pair_kind(c[0], c[1]);
    double r[3];
    for (int a = 0; a < 3; ++a) r[a] = q[a] - q[3 + a];
    const double s = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    double p, f[3];
    const int m = seg_ref(s, T.dx, T.n, p);
    cub3(term == 0 ? pr_rec(T, pk, m) + rho_off(pk, c[1]) : pr_rec(T, pk, m), p, f);
    const double cf = term == 0 ? n[1] : 0.5 * n[0] * n[1];
    hess_radial(r, s, f[1], f[2], (dir == 1 || dir == 2) ? -cf : cf, out);
    return;
  }
  if (!(dir == 0 || dir == 4 || dir == 5 || dir == 7 || dir == 8)) return;
  double r1[3], r2[3];
  for (int a = 0; a < 3; ++a) {
    r1[a] = q[a] - q[3 + a];
    r2[a] = q[a] - q[6 + a];
  }
  const double s1 = sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2]);
  const double s2 = sqrt(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2]);
  const double dd = r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2];
  const double c1 = n[0] * n[1], c2 = n[0] * n[2];
  double p1, p2, f1[3], f2[3];
  const int m1 = seg_ref(s1, T.dx, T.n, p1), m2 = seg_ref(s2, T.dx, T.n, p2);
  const int off = term == 2 ? 0 : 4;  // u or w in the segment record
  cub3(uw_rec(T, pair_kind(c[0], c[1]), m1) + off, p1, f1);
  cub3(uw_rec(T, pair_kind(c[0], c[2]), m2) + off, p2, f2);
  double H11[9] = {0}, H22[9] = {0}, H12[9] = {0};
  if (term == 2) {
    // 1/2 A1.A2 with A_k = c_k u(s_k) r_k
    double A1[3], A2[3];
    for (int a = 0; a < 3; ++a) {
      A1[a] = c1 * f1[0] * r1[a];
      A2[a] = c2 * f2[0] * r2[a];
    }
    auto vec = [&](const double *mv, const double *r, double s, const double (&f)[3], double cc,
                   double *H) {
      const double mr = mv[0] * r[0] + mv[1] * r[1] + mv[2] * r[2];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const double P = r[a] * r[b] / (s * s);
          H[3 * a + b] += cc * (f[1] * (mv[a] * r[b] + r[a] * mv[b]) / s +
                                mr * (f[2] * P + f[1] * ((a == b ? 1.0 : 0.0) - P) / s));
        }
    };
    vec(A2, r1, s1, f1, 0.5 * c1, H11);
    vec(A1, r2, s2, f2, 0.5 * c2, H22);
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) {
        double acc = 0.0;
        for (int z = 0; z < 3; ++z)
          acc += c1 * ((z == x ? f1[0] : 0.0) + f1[1] * r1[z] * r1[x] / s1) * c2 *
                 ((z == y ? f2[0] : 0.0) + f2[1] * r2[z] * r2[y] / s2);
        H12[3 * x + y] = 0.5 * acc;
      }
  } else {
    // 1/2 B1:B2 - 1/6 t1 t2 with B_k = c_k w(s_k) r_k r_k^T, t_k = c_k w(s_k) s_k^2
    const double t1 = c1 * f1[0] * s1 * s1, t2 = c2 * f2[0] * s2 * s2;
    const double hp1 = f1[1] * s1 * s1 + 2.0 * f1[0] * s1;
    const double hpp1 = f1[2] * s1 * s1 + 4.0 * f1[1] * s1 + 2.0 * f1[0];
    const double hp2 = f2[1] * s2 * s2 + 2.0 * f2[0] * s2;
    const double hpp2 = f2[2] * s2 * s2 + 4.0 * f2[1] * s2 + 2.0 * f2[0];
    auto ten = [&](const double *r_o, double c_o, double w_o, const double *r, double s,
                   const double (&f)[3], double cc, double *H) {
      // sum_ab M_ab d2 (w(s) r_a r_b) with M = c_o w_o r_o r_o^T
      double Mr[3];
      const double ro_r = r_o[0] * r[0] + r_o[1] * r[1] + r_o[2] * r[2];
      for (int a = 0; a < 3; ++a) Mr[a] = c_o * w_o * r_o[a] * ro_r;
      const double rMr = r[0] * Mr[0] + r[1] * Mr[1] + r[2] * Mr[2];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const double P = r[a] * r[b] / (s * s);
          H[3 * a + b] += cc * (rMr * (f[2] * P + f[1] * ((a == b ? 1.0 : 0.0) - P) / s) +
                                2.0 * f[1] * (r[a] * Mr[b] + Mr[a] * r[b]) / s +
                                2.0 * f[0] * c_o * w_o * r_o[a] * r_o[b]);
        }
    };
    ten(r2, c2, f2[0], r1, s1, f1, 0.5 * c1, H11);
    hess_radial(r1, s1, hp1, hpp1, -t2 * c1 / 6.0, H11);
    ten(r1, c1, f1[0], r2, s2, f2, 0.5 * c2, H22);
    hess_radial(r2, s2, hp2, hpp2, -t1 * c2 / 6.0, H22);
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) {
        const double G =
            c1 * c2 *
            (f1[1] * f2[1] * (r1[x] / s1) * (r2[y] / s2) * dd * dd +
             2.0 * f1[1] * f2[0] * (r1[x] / s1) * r1[y] * dd +
             2.0 * f1[0] * f2[1] * r2[x] * (r2[y] / s2) * dd +
             2.0 * f1[0] * f2[0] * ((x == y ? dd : 0.0) + r2[x] * r1[y]));
        const double g1 = c1 * hp1 * r1[x] / s1, g2 = c2 * hp2 * r2[y] / s2;
        H12[3 * x + y] = 0.5 * G - g1 * g2 / 6.0;
      }
  }
  for (int x = 0; x < 3; ++x)
    for (int y = 0; y < 3; ++y) {
      const int e = 3 * x + y, et = 3 * y + x;
      out[e] = dir == 0 ? H11[e] + H22[e] + H12[e] + H12[et]
               : dir == 4 ? H11[e] : dir == 8 ? H22[e] : dir == 5 ? H12[e] : H12[et];
    }
}

__global__ void __launch_bounds__(128) term_eval_kernel(TermArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  double q[9], n[3];
  int c[3];
  for (int e = 0; e < 9; ++e) q[e] = e < 3 * a.ns ? a.q[9 * (size_t)k + e] : 0.0;
  for (int s = 0; s < 3; ++s) {
    n[s] = s < a.ns ? a.x[3 * (size_t)k + s] : 0.0;
    c[s] = s < a.ns ? a.code[3 * (size_t)k + s] : 0;
  }
  double out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (a.fn == 0) {
    out[0] = term_F(a.T, a.term, c, n, q);
  } else if (a.fn == 1) {
    term_dq(a.T, a.term, c, n, a.dir, q, out);
  } else if (a.fn == 2) {
    term_d2(a.T, a.term, c, n, a.dir, q, out);
  } else if (a.fn == 3) {
    // dF_dq_FD: five points with step 1e-4 (1e-5 for the pair term,
    // dV_pair_ij_dq_FD) along each coordinate of slot dir; the moved
    // coordinate keeps its last position (+2 dr) while the next one moves,
    // as the reference's shared work array does
    const double dr = a.term == 1 ? 0.00001 : 0.0001;
    const double f0 = term_F(a.T, a.term, c, n, q);
    double qn[9];
    for (int e = 0; e < 9; ++e) qn[e] = q[e];
    for (int al = 0; al < 3; ++al) {
      const int d = a.dir * 3 + al;
      qn[d] = q[d] - dr * 2;
      const double fmm = term_F(a.T, a.term, c, n, qn);
      qn[d] = q[d] - dr;
      const double fm = term_F(a.T, a.term, c, n, qn);
      qn[d] = q[d] + dr;
      const double fp = term_F(a.T, a.term, c, n, qn);
      qn[d] = q[d] + dr * 2;
      const double fpp = term_F(a.T, a.term, c, n, qn);
      out[al] = ((fmm - f0) - 8.0 * (fm - f0) + 8.0 * (fp - f0) - (fpp - f0)) / (12.0 * dr);
    }
  } else if (a.fn == 4) {
    // d2F_dq2_FD: the diagonal entries only, second differences along the
    // coordinates of slot dir / (ns + 1); the quadrupole's fills blocks 0,
    // 4 and 8 only (dV2_quadrupole_ij1j2_dq2_FD)
    const double f0 = term_F(a.T, a.term, c, n, q);
    for (int al = 0; al < 3 && !(a.term == 3 && a.dir % 4 != 0); ++al) {
      const int d = a.dir / (1 + a.ns) * 3 + al;
      double s4[4];
      for (int w = 0; w < 4; ++w) {
        double qq[9];
        shifted(q, d, w, qq);
        s4[w] = term_F(a.T, a.term, c, n, qq);
      }
      out[4 * al] = d2_5(s4[0], s4[1], f0, s4[2], s4[3]);
    }
  } else {
    out[0] = term_dn(a.T, a.term, c, n, a.dir, q);
  }
  for (int e = 0; e < 9; ++e) a.out[9 * (size_t)k + e] = out[e];
}

// The same terms averaged over the reference's measure with the degree-3
// rule (meanfield_integral_gh3th, _gh_3th_dmq, _gh3th_dsq, _gh_3th_dxi,
// Quadrature-Hermitian-3th.cpp:36-378): mode 0 the value, 1 d/d mean q of
// slot dir (3 values), 2 d/d sigma of slot dir, 3 d/dx of slot dir.
__global__ void __launch_bounds__(128) term_quad_kernel(TermArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  double q[9], n[3], sig[3];
  int c[3];
  for (int e = 0; e < 9; ++e) q[e] = e < 3 * a.ns ? a.q[9 * (size_t)k + e] : 0.0;
  for (int s = 0; s < 3; ++s) {
    n[s] = s < a.ns ? a.x[3 * (size_t)k + s] : 0.0;
    sig[s] = s < a.ns ? a.sigma[3 * (size_t)k + s] : 0.0;
    c[s] = s < a.ns ? a.code[3 * (size_t)k + s] : 0;
  }
  const Gh3 m = gh3_of(a.ns, a.coincident != 0);
  const double W = 1.0 / (2.0 * m.D), zeta = sqrt((double)m.D) / kSqrt2d;
  double out[3] = {0, 0, 0};
  for (int sg = 0; sg < 2; ++sg)
    for (int l = 0; l < m.D; ++l) {
      const double sgn = sg == 0 ? 1.0 : -1.0;
      double ql[9];
      gh3_point(m, q, sig, l, sgn, ql);
      if (a.mode == 0) {
        out[0] += term_F(a.T, a.term, c, n, ql) * W;
      } else if (a.mode == 3) {
        out[0] += term_dn(a.T, a.term, c, n, a.dir, ql) * W;
      } else {
        double g[3];
        term_dq(a.T, a.term, c, n, a.dir, ql, g);
        for (int al = 0; al < 3; ++al) {
          if (a.mode == 1) {
            out[al] += g[al] * W;
          } else {
            const double b = (m.grp[a.dir] == l / 3 && al == l % 3) ? 1.0 : 0.0;
            out[0] += g[al] * (sgn * kSqrt2d * zeta * b) * W;
          }
        }
      }
    }
  for (int e = 0; e < 9; ++e) a.out[9 * (size_t)k + e] = e < 3 ? out[e] : 0.0;
}

// The reference's 5th-degree rule over the pair measure (Quadrature-
// Hermitian-5th.cpp:31-432; no caller in the reference selects it) of a
// pair term: mode 0 the average of F, 1 of dF_dq(dir), 2 of d2F_dq2(dir).
// 44 points, the 22 of its table and their negatives: z = (1, ..., 1)
// (weight 1/128), sqrt(2) e_k (k = 0..5; 1/16), (1, ..., 1) with entries a < b
// set to -1 (1/128); q = mean +- sqrt(2) sigma_s z, each value weighted
// W c0 with c0 = pi^(3/2), the sum scaled by pi^(-3/2), in that order.
__global__ void __launch_bounds__(128) term_quad5_kernel(TermArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  constexpr double kPi = 3.14159265358979323846;
  double q[9], n[3], sig[2];
  int c[3];
  for (int e = 0; e < 9; ++e) q[e] = e < 6 ? a.q[9 * (size_t)k + e] : 0.0;
  for (int s = 0; s < 3; ++s) {
    n[s] = s < 2 ? a.x[3 * (size_t)k + s] : 0.0;
    c[s] = s < 2 ? a.code[3 * (size_t)k + s] : 0;
  }
  sig[0] = a.sigma[3 * (size_t)k];
  sig[1] = a.sigma[3 * (size_t)k + 1];
  const double c0 = pow(sqrt(kPi), 6.0 / 2.0);
  const int nv = a.mode == 0 ? 1 : a.mode == 1 ? 3 : 9;
  double out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int sg = 0; sg < 2; ++sg)
    for (int gp = 0; gp < 22; ++gp) {
      // the point's entry z_m (m = 3 s + axis) and weight
      int pa = -1, pb = -1;
      if (gp >= 7) {  // pairs a < b in order
        int t = gp - 7;
        for (pa = 0; t >= 5 - pa; ++pa) t -= 5 - pa;
        pb = pa + 1 + t;
      }
      const double W = (gp >= 1 && gp <= 6) ? 0.0625 : 0.0078125;
      double ql[9];
      for (int e = 0; e < 9; ++e) ql[e] = 0.0;
      for (int al = 0; al < 3; ++al)
        for (int s = 0; s < 2; ++s) {
          const int m = 3 * s + al;
          const double z = gp == 0 ? 1.0
                         : gp <= 6 ? (m == gp - 1 ? kSqrt2d : 0.0)
                                   : ((m == pa || m == pb) ? -1.0 : 1.0);
          const double off = kSqrt2d * sig[s] * z;
          ql[m] = sg == 0 ? q[m] + off : q[m] - off;
        }
      double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (a.mode == 0) v[0] = term_F(a.T, a.term, c, n, ql);
      else if (a.mode == 1) term_dq(a.T, a.term, c, n, a.dir, ql, v);
      else term_d2(a.T, a.term, c, n, a.dir, ql, v);
      for (int e = 0; e < nv; ++e) out[e] += v[e] * W * c0;
    }
  const double sc = pow(1.0 / sqrt(kPi), 6.0 / 2.0);
  for (int e = 0; e < 9; ++e) a.out[9 * (size_t)k + e] = e < nv ? out[e] * sc : 0.0;
}

}  // namespace
}  // namespace btam

using namespace btam;

extern "C" {

int btam_mf_eval_multipole(btam_system *s, int rule, double *rho, double *V0, double *S0,
                           double *energy) {
  if (!s || (rule != BTAM_MP_FD && rule != BTAM_MP_ANALYTIC)) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const size_t n = (size_t)s->n_real;
  double *rd = nullptr, *vd = nullptr, *sd = nullptr;
  BTAM_TRY(dalloc(rd, s->st, n));
  int st = dalloc(vd, s->st, n);
  if (st == BTAM_OK) st = dalloc(sd, s->st, n);
  if (st != BTAM_OK) {
    dfree(rd, s->st);
    dfree(vd, s->st);
    return st;
  }
  MpArgs a;
  a.n_real = s->n_real;
  a.rule = rule;
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.offs = s->offs;
  a.idx = s->idx;
  a.T = s->T->r64;
  a.emb_mg = s->T->v64.t[T_F_MG];
  a.emb_h = s->T->v64.t[T_F_H];
  a.rho = rd;
  a.S0 = nullptr;
  a.gamma = s->gamma;
  a.mass[0] = tables_mass(s->T, 0);
  a.mass[1] = tables_mass(s->T, 1);
  const int g = (int)(((long long)s->n_real * 32 + 127) / 128);
  cudaError_t e = cudaSuccess;
  if (g > 0) {
    a.out = rd;
    mp_rho_kernel<<<g, 128, 0, s->st>>>(a);
    a.out = vd;
    a.S0 = sd;
    mp_v0_kernel<<<g, 128, 0, s->st>>>(a);
    e = cudaGetLastError();
  }
  std::vector<double> hv(n);
  if (e == cudaSuccess && rho && n)
    e = cudaMemcpyAsync(rho, rd, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess && S0 && n)
    e = cudaMemcpyAsync(S0, sd, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess && n)
    e = cudaMemcpyAsync(hv.data(), vd, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  dfree(rd, s->st);
  dfree(vd, s->st);
  dfree(sd, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  double E = 0.0;
  for (size_t k = 0; k < n; ++k) E += hv[k];
  if (V0) std::copy(hv.begin(), hv.end(), V0);
  if (energy) *energy = E;
  return read_err(s);
}

}  // extern "C"

namespace {

// The multipole residuals (Rq, Rs, Rx; any may be null) and, when self5 or
// slot5 is given, their unweighted per-pair terms split out of the pairs
// kernel's buffer (per real site u: entry 0 the pair (u, u), entries 1.. its
// list entries in order): self5 (5 per real site), slot5 (5 per list entry;
// slot_cap entries at least).
int mp_residuals(btam_system *s, int rule, double *Rq, double *Rs, double *Rx, double *self5,
                 double *slot5, long long slot_cap) {
  if (!s || (rule != BTAM_MP_FD && rule != BTAM_MP_ANALYTIC)) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const size_t n = (size_t)s->n_real;
  if (n == 0) return BTAM_OK;
  std::vector<int> offs_n(1);
  cudaError_t e = cudaMemcpyAsync(offs_n.data(), s->offs + n, sizeof(int),
                                  cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) return cuda_status(e);
  if (slot5 && slot_cap < offs_n[0]) return BTAM_ERR_ARG;
  const long long total = (long long)offs_n[0] + (long long)n;
  double *rd = nullptr, *g5 = nullptr, *gk = nullptr, *out = nullptr;
  BTAM_TRY(dalloc(rd, s->st, n));
  int st = dalloc(g5, s->st, 5 * (size_t)total);
  if (st == BTAM_OK) st = dalloc(gk, s->st, 5 * (size_t)total);
  if (st == BTAM_OK) st = dalloc(out, s->st, 5 * n);
  if (st != BTAM_OK) {
    dfree(rd, s->st);
    dfree(g5, s->st);
    dfree(gk, s->st);
    return st;
  }
  MpResArgs r;
  MpArgs &a = r.b;
  a.n_real = s->n_real;
  a.rule = rule;
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.offs = s->offs;
  a.idx = s->idx;
  a.T = s->T->r64;
  a.emb_mg = s->T->v64.t[T_F_MG];
  a.emb_h = s->T->v64.t[T_F_H];
  a.rho = rd;
  a.out = rd;
  a.S0 = nullptr;
  a.gamma = s->gamma;
  a.mass[0] = tables_mass(s->T, 0);
  a.mass[1] = tables_mass(s->T, 1);
  r.owner = s->owner;
  r.rev = s->rev;
  r.gamma = s->gamma;
  r.gk = gk;
  r.g5 = g5;
  r.Rq = out;
  r.Rs = out + 3 * n;
  r.Rx = out + 4 * n;
  const int g = (int)(((long long)n * 32 + 127) / 128);
  mp_rho_kernel<<<g, 128, 0, s->st>>>(a);
  mp_centre_kernel<<<(int)((n + kMpW - 1) / kMpW), kMpW * 32, 0, s->st>>>(r);
  mp_gather_kernel<<<g, 128, 0, s->st>>>(r);
  mp_assemble_kernel<<<(int)((n + 127) / 128), 128, 0, s->st>>>(r);
  e = cudaGetLastError();
  if (e == cudaSuccess && Rq)
    e = cudaMemcpyAsync(Rq, out, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess && Rs)
    e = cudaMemcpyAsync(Rs, out + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess && Rx)
    e = cudaMemcpyAsync(Rx, out + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  std::vector<double> g5h, offsh;
  std::vector<int> offs_h;
  if (e == cudaSuccess && (self5 || slot5)) {
    g5h.resize(5 * (size_t)total);
    offs_h.resize(n + 1);
    e = cudaMemcpyAsync(g5h.data(), g5, g5h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                        s->st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(offs_h.data(), s->offs, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                          s->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e == cudaSuccess && (self5 || slot5)) {
    for (size_t u = 0; u < n; ++u) {
      const double *g = g5h.data() + 5 * ((size_t)offs_h[u] + u);
      if (self5)
        for (int c = 0; c < 5; ++c) self5[5 * u + c] = g[c];
      if (slot5)
        for (int p = offs_h[u]; p < offs_h[u + 1]; ++p)
          for (int c = 0; c < 5; ++c) slot5[5 * (size_t)p + c] = g[5 * (1 + p - offs_h[u]) + c];
    }
  }
  dfree(rd, s->st);
  dfree(g5, s->st);
  dfree(gk, s->st);
  dfree(out, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  return read_err(s);
}

}  // namespace

extern "C" {

int btam_mf_residuals_multipole(btam_system *s, int rule, double *Rq, double *Rs, double *Rx) {
  if (!Rq || !Rs || !Rx) return BTAM_ERR_ARG;
  return mp_residuals(s, rule, Rq, Rs, Rx, nullptr, nullptr, 0);
}

int btam_mf_pair_terms_multipole(btam_system *s, int rule, double *self, double *slot,
                                 long long slot_cap) {
  return mp_residuals(s, rule, nullptr, nullptr, nullptr, self, slot, slot_cap);
}

int btam_mf_stress_multipole(btam_system *s, int rule, double *W0, double *total) {
  if (!s || (rule != BTAM_MP_FD && rule != BTAM_MP_ANALYTIC)) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const size_t n = (size_t)s->n_real;
  double *rd = nullptr, *wd = nullptr;
  BTAM_TRY(dalloc(rd, s->st, n));
  int st = dalloc(wd, s->st, 9 * n);
  if (st != BTAM_OK) {
    dfree(rd, s->st);
    return st;
  }
  MpArgs a;
  a.n_real = s->n_real;
  a.rule = rule;
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.offs = s->offs;
  a.idx = s->idx;
  a.T = s->T->r64;
  a.emb_mg = s->T->v64.t[T_F_MG];
  a.emb_h = s->T->v64.t[T_F_H];
  a.rho = rd;
  a.out = rd;
  a.S0 = nullptr;
  a.gamma = s->gamma;
  a.mass[0] = tables_mass(s->T, 0);
  a.mass[1] = tables_mass(s->T, 1);
  const int g = (int)(((long long)n * 32 + 127) / 128);
  cudaError_t e = cudaSuccess;
  std::vector<double> hw(9 * n);
  if (g > 0) {
    mp_rho_kernel<<<g, 128, 0, s->st>>>(a);
    mp_stress_kernel<<<g, 128, 0, s->st>>>(a, wd);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hw.data(), wd, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  dfree(rd, s->st);
  dfree(wd, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  if (W0) std::copy(hw.begin(), hw.end(), W0);
  if (total) {
    for (int c = 0; c < 9; ++c) total[c] = 0.0;
    for (size_t k = 0; k < n; ++k)
      for (int c = 0; c < 9; ++c) total[c] += hw[9 * k + c];
  }
  return read_err(s);
}

}  // extern "C"

namespace {

// The multipole Hessian blocks: H (9 per real site, may be null) summed over
// i in {u} U N(u), or with Hslot (9 per list entry; slot_cap entries at
// least) the i = u blocks in H and the per-neighbour blocks in Hslot.
int mp_hessian(btam_system *s, int rule, double *H, double *Hslot, long long slot_cap) {
  if (!s || (rule != BTAM_MP_FD && rule != BTAM_MP_ANALYTIC)) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const size_t n = (size_t)s->n_real;
  if (n == 0) return BTAM_OK;
  int np = 0;
  cudaError_t e = cudaMemcpyAsync(&np, s->offs + n, sizeof(int), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) return cuda_status(e);
  if (Hslot && slot_cap < np) return BTAM_ERR_ARG;
  double *rd = nullptr, *G = nullptr, *Hd = nullptr, *Hs = nullptr;
  BTAM_TRY(dalloc(rd, s->st, n));
  int st = dalloc(G, s->st, 3 * (size_t)(np > 0 ? np : 1));
  if (st == BTAM_OK) st = dalloc(Hd, s->st, 9 * n);
  if (st == BTAM_OK && Hslot) st = dalloc(Hs, s->st, 9 * (size_t)(np > 0 ? np : 1));
  if (st != BTAM_OK) {
    dfree(rd, s->st);
    dfree(G, s->st);
    dfree(Hd, s->st);
    return st;
  }
  MpArgs a;
  a.n_real = s->n_real;
  a.rule = rule;
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.offs = s->offs;
  a.idx = s->idx;
  a.T = s->T->r64;
  a.emb_mg = s->T->v64.t[T_F_MG];
  a.emb_h = s->T->v64.t[T_F_H];
  a.rho = rd;
  a.out = rd;
  a.S0 = nullptr;
  a.gamma = s->gamma;
  a.mass[0] = tables_mass(s->T, 0);
  a.mass[1] = tables_mass(s->T, 1);
  const int g = (int)(((long long)n * 32 + 127) / 128);
  mp_rho_kernel<<<g, 128, 0, s->st>>>(a);
  mp_rho_grad_kernel<<<g, 128, 0, s->st>>>(a, G);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    st = mf_hessian_enqueue_with(s, rd, G, Hd, Hs);
    if (st == BTAM_OK && H)
      e = cudaMemcpyAsync(H, Hd, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
    if (st == BTAM_OK && e == cudaSuccess && Hslot)
      e = cudaMemcpyAsync(Hslot, Hs, 9 * (size_t)np * sizeof(double), cudaMemcpyDeviceToHost,
                          s->st);
    if (st == BTAM_OK && e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  }
  dfree(rd, s->st);
  dfree(G, s->st);
  dfree(Hd, s->st);
  dfree(Hs, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  if (st != BTAM_OK) return st;
  return read_err(s);
}

}  // namespace

extern "C" {

int btam_mf_hessian_multipole(btam_system *s, int rule, double *H) {
  if (!H) return BTAM_ERR_ARG;
  return mp_hessian(s, rule, H, nullptr, 0);
}

int btam_mf_hessian_pairs_multipole(btam_system *s, int rule, double *Hself, double *Hslot,
                                    long long slot_cap) {
  if (!Hself || !Hslot) return BTAM_ERR_ARG;
  return mp_hessian(s, rule, Hself, Hslot, slot_cap);
}

}  // extern "C"

// ---- the per-term plugin interface (C ABI) ----------------------------------
namespace {

int term_launch(const btam_tables *t, bool quad, int term, int fn_or_mode, int dir, int slot_ns,
                int coincident, int n, const double *q, const double *sigma, const double *x,
                const int *species, double *out, bool fifth = false) {
  if (!t || n < 0 || !q || !x || !species || !out || ((quad || fifth) && !sigma))
    return BTAM_ERR_ARG;
  if (term < 0 || term > 3) return BTAM_ERR_ARG;
  const int ns = term < 2 ? 2 : 3;
  if (slot_ns != ns) return BTAM_ERR_ARG;
  if (quad ? (fn_or_mode < 0 || fn_or_mode > 3) : (fn_or_mode < 0 || fn_or_mode > 5))
    return BTAM_ERR_ARG;
  const bool block = !quad && (fn_or_mode == 2 || fn_or_mode == 4);
  if (fn_or_mode != 0 && (dir < 0 || dir >= (block ? ns * ns : ns))) return BTAM_ERR_ARG;
  if (n == 0) return BTAM_OK;
  std::vector<int> code(3 * (size_t)n, 0);
  for (size_t k = 0; k < 3 * (size_t)n; ++k) {
    if (k % 3 >= (size_t)ns) continue;
    if (species[k] == 12) code[k] = 0;
    else if (species[k] == 1) code[k] = 1;
    else return BTAM_ERR_SPECIES;
  }
  cudaStream_t st = cudaStreamPerThread;
  double *dq = nullptr, *dx = nullptr, *ds = nullptr, *dout = nullptr;
  int *dc = nullptr;
  cudaError_t e = dalloc(dq, st, 9 * (size_t)n);
  if (e == cudaSuccess) e = dalloc(dx, st, 3 * (size_t)n);
  if (e == cudaSuccess) e = dalloc(ds, st, 3 * (size_t)n);
  if (e == cudaSuccess) e = dalloc(dout, st, 9 * (size_t)n);
  if (e == cudaSuccess) e = dalloc(dc, st, 3 * (size_t)n);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dq, q, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dx, x, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && (quad || fifth))
    e = cudaMemcpyAsync(ds, sigma, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dc, code.data(), 3 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    TermArgs a;
    a.T = t->r64;
    a.term = term;
    a.fn = quad ? 0 : fn_or_mode;
    a.mode = (quad || fifth) ? fn_or_mode : 0;
    a.dir = dir;
    a.ns = ns;
    a.n = n;
    a.coincident = coincident;
    a.q = dq;
    a.x = dx;
    a.sigma = ds;
    a.code = dc;
    a.out = dout;
    const int g = (n + 127) / 128;
    if (fifth) term_quad5_kernel<<<g, 128, 0, st>>>(a);
    else if (quad) term_quad_kernel<<<g, 128, 0, st>>>(a);
    else term_eval_kernel<<<g, 128, 0, st>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, dout, 9 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  dfree(dq, st);
  dfree(dx, st);
  dfree(ds, st);
  dfree(dout, st);
  dfree(dc, st);
  return cuda_status(e);
}

}  // namespace

extern "C" {

int btam_term_eval(const btam_tables *t, int term, int fn, int direction, int n,
                   const double *q, const double *x, const int *species, double *out) {
  return term_launch(t, false, term, fn, direction, term < 2 ? 2 : 3, 0, n, q, nullptr, x,
                     species, out);
}

int btam_term_quadrature5(const btam_tables *t, int term, int mode, int direction, int n,
                          const double *q, const double *sigma, const double *x,
                          const int *species, double *out) {
  if (term < 0 || term > 1 || mode < 0 || mode > 2) return BTAM_ERR_ARG;
  if (mode > 0 && (direction < 0 || direction >= (mode == 1 ? 2 : 4))) return BTAM_ERR_ARG;
  // the term evaluator's argument checks with the slot function of the mode
  return term_launch(t, false, term, mode == 0 ? 0 : mode == 1 ? 1 : 2, mode == 0 ? 0 : direction,
                     2, 0, n, q, sigma, x, species, out, true);
}

int btam_term_quadrature(const btam_tables *t, int term, int mode, int slot, int coincident,
                         int n, const double *q, const double *sigma, const double *x,
                         const int *species, double *out) {
  if (coincident && term < 2) return BTAM_ERR_ARG;
  return term_launch(t, true, term, mode, slot, term < 2 ? 2 : 3, coincident, n, q, sigma, x,
                     species, out);
}

}  // extern "C"
