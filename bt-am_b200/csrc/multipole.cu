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
namespace {

// cubic_spline (cubic-spline.cpp:84-96) in the reference's operation order:
// m = min((int)(x / dx), n - 1), p = min(x - m dx, dx).
__device__ __forceinline__ int seg_ref(double x, double dx, int n, double &p) {
  int m = (int)(x / dx);
  m = m < n - 1 ? m : n - 1;
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
__device__ TriTr tri_traces(const RadialView<double> &T, int pk1, int pk2, const double *n,
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
  }
}

}  // namespace
}  // namespace btam

using namespace btam;

extern "C" {

int btam_mf_eval_multipole(btam_system *s, int rule, double *rho, double *V0, double *energy) {
  if (!s || (rule != BTAM_MP_FD && rule != BTAM_MP_ANALYTIC)) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const size_t n = (size_t)s->n_real;
  double *rd = nullptr, *vd = nullptr;
  BTAM_TRY(dalloc(rd, s->st, n));
  int st = dalloc(vd, s->st, n);
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
  const int g = (int)(((long long)s->n_real * 32 + 127) / 128);
  cudaError_t e = cudaSuccess;
  if (g > 0) {
    a.out = rd;
    mp_rho_kernel<<<g, 128, 0, s->st>>>(a);
    a.out = vd;
    mp_v0_kernel<<<g, 128, 0, s->st>>>(a);
    e = cudaGetLastError();
  }
  std::vector<double> hv(n);
  if (e == cudaSuccess && rho && n)
    e = cudaMemcpyAsync(rho, rd, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess && n)
    e = cudaMemcpyAsync(hv.data(), vd, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  dfree(rd, s->st);
  dfree(vd, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  double E = 0.0;
  for (size_t k = 0; k < n; ++k) E += hv[k];
  if (V0) std::copy(hv.begin(), hv.end(), V0);
  if (energy) *energy = E;
  return read_err(s);
}

}  // extern "C"
