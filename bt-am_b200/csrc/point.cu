// Non-mean-field forms of the ADP (the sigma -> 0 limit: every term at the
// mean positions) and the bulk stretch relaxation that consumes them.
//
// The reference evaluates these one (u, i) pair at a time with the triplet
// double loop over N(i) (evaluate_DV_i_Dq_u_adp_MgHx, MgHx-mf-V-bulk.cpp:
// 147-330; evaluate_DV_i_dF_MgHx, 530-704).  Summed over j1, j2 with the
// factor 2 of j1 != j2, the dipole and quadrupole terms of site i are
//   1/2 |mu_i|^2 + 1/2 |Lambda_i|_F^2 - 1/6 (tr Lambda_i)^2,
//   mu_i = sum_j x_i x_j u(r_ij) r_ij,  Lambda_i = sum_j x_i x_j w(r_ij) r_ij r_ij^T,
// so two passes over the neighbour lists give every derivative:
//   pass 1 (pt_moments_kernel): per site rho_i, x_i F'(rho_i), mu_i,
//           Lambda_i, tr Lambda_i and the point energy V_i (a 16-double
//           record);
//   pass 2 (pt_grad_kernel): per real site u and neighbour j the gradient
//           g(u->j) = dV_u/dq_j from u's record and h(j->u) = dV_j/dq_u from
//           the record of j's owner (the moments are translation invariant,
//           so a periodic image shares its owner's record):
//             Fq_u = sum_j h(j->u) - g(u->j)   (= sum_{i in {u} U N(u)} dV_i/dq_u)
//             W_u  = sum_j g(u->j) (x) (q_j - q_u)
//           W_u is dV_u/dF (row: gradient component, column: position
//           component) taken at q0 = q; by translation invariance of V_u it
//           equals the reference's sum over the term sites a of
//           dV_u/dq_a (x) q0_a.
// A lane per neighbour, a warp per site, fixed-order warp reductions: the
// results are deterministic.
#include <cmath>
#include <functional>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "linalg.hpp"
#include "ngmres.hpp"

namespace btam {
namespace {

constexpr int kPtRec = 16;    // record: rho, xF', mu (3), Lambda (xx yy zz yz xz xy), tr, V, 0 0 0
constexpr int kPtParts = 64;  // first-stage partial sums of the totals
constexpr int kPtTot = 12;    // totals: sum V, sum |Fq|^2, sum W (9, row-major), 0

struct PtArgs {
  int n_real;
  const double4 *pos;
  const double2 *xb;
  const int *code, *owner, *offs, *idx;
  RadialView<double> T;
  SplineView<double> emb_mg, emb_h;
  double *rec, *rho, *V, *Fq, *W;
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// A site record: 128 bytes, 128-byte aligned, four 256-bit loads.
__device__ __forceinline__ void ld_rec(const double *r, double (&a)[kPtRec]) {
  double lo[8], hi[8];
  ld8(r, lo);
  ld8(r + 8, hi);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    a[k] = lo[k];
    a[8 + k] = hi[k];
  }
}
// Its first 12 values (rho .. tr Lambda), all a gradient needs: three
// 256-bit loads.
__device__ __forceinline__ void ld_rec12(const double *r, double (&a)[kPtRec]) {
  double lo[8], hi[4];
  ld8(r, lo);
  ld4(r + 8, hi);
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = lo[k];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[8 + k] = hi[k];
#pragma unroll
  for (int k = 12; k < kPtRec; ++k) a[k] = 0.0;
}

// Pass 1: rho_i = sum_j x_j rho_{s_j}(r) (evaluate_rho_i_adp_MgHx,
// MgHx-mf-V-bulk.cpp:83-143), the moments and the point energy.  Neighbours
// with x_j < min_occupancy are skipped (a Mg neighbour can only be empty at
// x = 0, where its terms vanish, so the reference's H-only tests of
// 200-202 and 252-254 give the same sums).
__global__ void __launch_bounds__(128) pt_moments_kernel(PtArgs a) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.n_real) return;
  const double xi = a.xb[i].x;
  const int ci = a.code[i];
  double acc[11];
#pragma unroll
  for (int c = 0; c < 11; ++c) acc[c] = 0.0;
  if (!(xi < kMinOcc)) {
    const double4 qi = a.pos[i];
    for (int p = a.offs[i] + lane; p < a.offs[i + 1]; p += 32) {
      const int j = a.idx[p];
      const double xj = a.xb[j].x;
      if (xj < kMinOcc) continue;
      const double4 qj = a.pos[j];
      const int cj = a.code[j], pk = pair_kind(ci, cj);
      const V3<double> r = mk3<double>(qj.x - qi.x, qj.y - qi.y, qj.z - qi.z);
      Geo<double> g;
      double pp, ph, dph, rj, drj, ri, dri;
      const int m = geo_uw<double, false>(g, r, a.T, pk, pp);
      pr_at<double, false, false>(a.T, pk, ci, cj, m, pp, ph, dph, rj, drj, ri, dri);
      const double t = xi * xj, tu = t * g.u, tw = t * g.w;
      acc[0] += xj * rj;
      acc[1] += 0.5 * (t * ph);
      acc[2] += tu * r.x;
      acc[3] += tu * r.y;
      acc[4] += tu * r.z;
      acc[5] += tw * r.x * r.x;
      acc[6] += tw * r.y * r.y;
      acc[7] += tw * r.z * r.z;
      acc[8] += tw * r.y * r.z;
      acc[9] += tw * r.x * r.z;
      acc[10] += tw * r.x * r.y;
    }
  }
#pragma unroll
  for (int c = 0; c < 11; ++c) acc[c] = wsum(acc[c]);
  if (lane == 0) {
    double F = 0.0, dF = 0.0;
    if (!(xi < kMinOcc)) spline_vd(ci == 0 ? a.emb_mg : a.emb_h, acc[0], F, dF);
    const double tr = acc[5] + acc[6] + acc[7];
    const double mm = acc[2] * acc[2] + acc[3] * acc[3] + acc[4] * acc[4];
    const double ll = acc[5] * acc[5] + acc[6] * acc[6] + acc[7] * acc[7] +
                      2.0 * (acc[8] * acc[8] + acc[9] * acc[9] + acc[10] * acc[10]);
    const double V = (xi < kMinOcc) ? 0.0 : xi * F + acc[1] + 0.5 * mm + 0.5 * ll - tr * tr / 6.0;
    double4 *o = reinterpret_cast<double4 *>(a.rec + (size_t)kPtRec * i);
    o[0] = make_double4(acc[0], xi * dF, acc[2], acc[3]);
    o[1] = make_double4(acc[4], acc[5], acc[6], acc[7]);
    o[2] = make_double4(acc[8], acc[9], acc[10], tr);
    o[3] = make_double4(V, 0.0, 0.0, 0.0);
    a.rho[i] = acc[0];
    a.V[i] = V;
  }
}

// Gradient of V_c with respect to the neighbour at r = q_nb - q_c, from c's
// record m: the embedding, pair, dipole and quadrupole terms of
// MgHx-ADP.cpp:557-601, 904-949, 1285-1371, 1835-1935 summed over the
// triplets through the moments.  t = x_c x_nb, drho = rho'_{s_nb}(s).
__device__ __forceinline__ V3<double> pt_grad(const double (&m)[kPtRec], const V3<double> &r,
                                              const Geo<double> &g, double t, double x_nb,
                                              double drho, double dph) {
  const V3<double> mu = mk3<double>(m[2], m[3], m[4]);
  const V3<double> Lr = mk3<double>(m[5] * r.x + m[10] * r.y + m[9] * r.z,
                                    m[10] * r.x + m[6] * r.y + m[8] * r.z,
                                    m[9] * r.x + m[8] * r.y + m[7] * r.z);
  const double cr = m[1] * x_nb * drho + 0.5 * (t * dph) + t * g.du * dot3(mu, r) +
                    t * g.dw * dot3(r, Lr);
  const double ca = t * g.u, cl = 2.0 * t * g.w;
  const double cv = -(m[11] * t * (g.dw * g.s + 2.0 * g.w)) / 3.0;
  const double k = cr * g.inv_s + cv;
  return mk3<double>(k * r.x + ca * mu.x + cl * Lr.x, k * r.y + ca * mu.y + cl * Lr.y,
                     k * r.z + ca * mu.z + cl * Lr.z);
}

// PAIRS: the per-pair terms instead of their sum: slot3[3p..] = h(j->u) =
// dV_j/dq_u for every entry p of u's list (0 for an empty j) and Fq_u =
// -sum_j g(u->j) = dV_u/dq_u (evaluate_DV_i_Dq_u_adp_MgHx at (u, j) and
// (u, u)).
template <bool PAIRS>
__global__ void __launch_bounds__(128) pt_grad_kernel(PtArgs a, double *slot3) {
  const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= a.n_real) return;
  const double xu = a.xb[u].x;
  const int cu = a.code[u];
  double acc[12];
#pragma unroll
  for (int c = 0; c < 12; ++c) acc[c] = 0.0;
  if (PAIRS && xu < kMinOcc)
    for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32)
      for (int c = 0; c < 3; ++c) slot3[3 * (size_t)p + c] = 0.0;
  if (!(xu < kMinOcc)) {
    double mu_[kPtRec];
    ld_rec(a.rec + (size_t)kPtRec * u, mu_);
    const double4 qu = a.pos[u];
    for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32) {
      const int j = a.idx[p];
      const double xj = a.xb[j].x;
      if (PAIRS && xj < kMinOcc)
        for (int c = 0; c < 3; ++c) slot3[3 * (size_t)p + c] = 0.0;
      if (xj < kMinOcc) continue;
      const double4 qj = a.pos[j];
      const int cj = a.code[j], pk = pair_kind(cu, cj);
      const V3<double> r = mk3<double>(qj.x - qu.x, qj.y - qu.y, qj.z - qu.z);
      Geo<double> g;
      double pp, ph, dph, rj, drj, ru, dru;
      const int m = geo_uw<double, true>(g, r, a.T, pk, pp);
      pr_at<double, true, true>(a.T, pk, cu, cj, m, pp, ph, dph, rj, drj, ru, dru);
      const double t = xu * xj;
      const V3<double> gu = pt_grad(mu_, r, g, t, xj, drj, dph);
      double mo[kPtRec];
      ld_rec12(a.rec + (size_t)kPtRec * a.owner[j], mo);
      const V3<double> rn = mk3<double>(-r.x, -r.y, -r.z);
      const V3<double> hj = pt_grad(mo, rn, g, t, xu, dru, dph);
      if (PAIRS) {
        slot3[3 * (size_t)p] = hj.x;
        slot3[3 * (size_t)p + 1] = hj.y;
        slot3[3 * (size_t)p + 2] = hj.z;
        acc[0] -= gu.x;
        acc[1] -= gu.y;
        acc[2] -= gu.z;
      } else {
        acc[0] += hj.x - gu.x;
        acc[1] += hj.y - gu.y;
        acc[2] += hj.z - gu.z;
      }
      acc[3] += gu.x * r.x;
      acc[4] += gu.x * r.y;
      acc[5] += gu.x * r.z;
      acc[6] += gu.y * r.x;
      acc[7] += gu.y * r.y;
      acc[8] += gu.y * r.z;
      acc[9] += gu.z * r.x;
      acc[10] += gu.z * r.y;
      acc[11] += gu.z * r.z;
    }
  }
#pragma unroll
  for (int c = 0; c < 12; ++c) acc[c] = wsum(acc[c]);
  if (lane == 0) {
    for (int c = 0; c < 3; ++c) a.Fq[3 * (size_t)u + c] = acc[c];
    for (int c = 0; c < 9; ++c) a.W[9 * (size_t)u + c] = acc[3 + c];
  }
}

// ---- Hessian blocks of the point forms (evaluate_D2V_i_Dq2_u_MgHx,
// MgHx-mf-V-bulk.cpp:333-528), summed over i in {u} U N(u).  Through the
// moments (r = q_nb - q_c, P = r r^T / s^2, Q = (I - P) / s):
//   i = u: the full Hessian of V_u in q_u,
//     x F'' g g^T + K^T K + sum_ab dLambda_ab dLambda_ab^T - 1/3 T T^T   (pass 1b)
//     + per neighbour, linear in u's record (pass 2b):
//       e x_j rho_j-Hessian + 1/2 t phi-Hessian + mu . d2(a_j) + Lambda : d2(b_j)
//       - 1/3 tr Lambda d2(tr b_j),
//     g = sum drho/dq, K = dmu/dq, dLambda/dq, T = d tr Lambda/dq;
//   i = neighbour j: the reference sums the diagonal slot blocks of u in
//     V_j's terms, whose triplet parts are linear in j's moments (for
//     j1 = j2 = u it adds the two slot blocks without their cross blocks):
//       x_j F''(rho_j) (x_u rho_u')^2 P + e_j x_u rho_u-Hessian + 1/2 t phi-Hessian
//       + mu_j . d2(a_u) + Lambda_j : d2(b_u) - 1/3 tr Lambda_j d2(tr b_u).
// a = t u(s) r, b = t w(s) r r^T with t = x_c x_nb.

// Spline value and first and second derivatives of a segment record.
__device__ __forceinline__ void cub_vdd(const double *k, double p, double &v, double &d1,
                                        double &d2) {
  v = k[0] + (k[1] + (k[2] + k[3] * p) * p) * p;
  d1 = k[1] + (2.0 * k[2] + 3.0 * k[3] * p) * p;
  d2 = 2.0 * k[2] + 6.0 * k[3] * p;
}

struct PtSpl {
  double s, u, du, ddu, w, dw, ddw, ph, dph, ddph;
  double rn, drn, ddrn;  // rho of the neighbour's species
  double rc, drc, ddrc;  // rho of the centre's species
};

// Every spline of pair kind pk at |r| = s, with second derivatives.
__device__ __forceinline__ PtSpl pt_splines(const RadialView<double> &T, int pk, int cc, int cn,
                                            double s) {
  PtSpl o;
  o.s = s;
  double p;
  const int m = seg_of(T, s, p);
  double k[8];
  ld8(uw_rec(T, pk, m), k);
  cub_vdd(k, p, o.u, o.du, o.ddu);
  cub_vdd(k + 4, p, o.w, o.dw, o.ddw);
  const double *pr = pr_rec(T, pk, m);
  double h[8];
  ld8(pr, h);
  cub_vdd(h, p, o.ph, o.dph, o.ddph);
  double hr[4];
  const int on = rho_off(pk, cn), oc = rho_off(pk, cc);
  for (int c = 0; c < 4; ++c) hr[c] = pr[on + c];
  cub_vdd(hr, p, o.rn, o.drn, o.ddrn);
  for (int c = 0; c < 4; ++c) hr[c] = pr[oc + c];
  cub_vdd(hr, p, o.rc, o.drc, o.ddrc);
  return o;
}

// Symmetric 3x3 as xx yy zz yz xz xy.
__device__ __forceinline__ int sym6(int a, int b) {
  return a == b ? a : (a + b == 3 ? 3 : (a + b == 2 ? 4 : 5));
}

// Adds the terms linear in a centre's record m (e = x_c F'(rho_c), mu,
// Lambda, tr Lambda) for the neighbour at r, plus f P with the given radial
// coefficients: c_rad = the coefficient pair (c'', c') of P and Q.
__device__ __forceinline__ void pt_hess_linear(const double (&m)[kPtRec], const double *r,
                                               const PtSpl &S, double t, double cpp,
                                               double cp, double (&H)[6]) {
  const double s = S.s, is = 1.0 / s;
  const double mu[3] = {m[2], m[3], m[4]};
  const double L[9] = {m[5], m[10], m[9], m[10], m[6], m[8], m[9], m[8], m[7]};
  double Lr[3];
  for (int a = 0; a < 3; ++a) Lr[a] = L[3 * a] * r[0] + L[3 * a + 1] * r[1] + L[3 * a + 2] * r[2];
  const double mr = mu[0] * r[0] + mu[1] * r[1] + mu[2] * r[2];
  const double rLr = r[0] * Lr[0] + r[1] * Lr[1] + r[2] * Lr[2];
  const double hp = S.dw * s * s + 2.0 * S.w * s, hpp = S.ddw * s * s + 4.0 * S.dw * s + 2.0 * S.w;
  // coefficients of P and Q
  const double cP = cpp + t * mr * S.ddu + t * rLr * S.ddw - m[11] * t * hpp / 3.0;
  const double cQ = cp + t * mr * S.du + t * rLr * S.dw - m[11] * t * hp / 3.0;
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      const double P = r[a] * r[b] * is * is;
      const double Q = ((a == b ? 1.0 : 0.0) - P) * is;
      H[sym6(a, b)] += cP * P + cQ * Q + t * S.du * (mu[a] * r[b] + r[a] * mu[b]) * is +
                       2.0 * t * S.dw * (r[a] * Lr[b] + Lr[a] * r[b]) * is +
                       2.0 * t * S.w * L[3 * a + b];
    }
}

// Pass 1b: the self products of site i and x_i F''(rho_i) into hrec (8 per
// site: x F'', then the six entries of x F'' g g^T + K^T K + sum dL dL^T -
// T T^T / 3).
__global__ void __launch_bounds__(128) pt_hself_kernel(PtArgs a, double *hrec) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= a.n_real) return;
  const double xi = a.xb[i].x;
  const int ci = a.code[i];
  // g (3), K (6 sym), dLambda (6 entries x 3), T (3)
  double acc[30];
#pragma unroll
  for (int c = 0; c < 30; ++c) acc[c] = 0.0;
  if (!(xi < kMinOcc)) {
    const double4 qi = a.pos[i];
    for (int p = a.offs[i] + lane; p < a.offs[i + 1]; p += 32) {
      const int j = a.idx[p];
      const double xj = a.xb[j].x;
      if (xj < kMinOcc) continue;
      const double4 qj = a.pos[j];
      const int cj = a.code[j], pk = pair_kind(ci, cj);
      const double r[3] = {qj.x - qi.x, qj.y - qi.y, qj.z - qi.z};
      const double s = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]), is = 1.0 / s;
      const PtSpl S = pt_splines(a.T, pk, ci, cj, s);
      const double t = xi * xj;
      for (int c = 0; c < 3; ++c) acc[c] += xj * S.drn * r[c] * is;
      for (int x = 0; x < 3; ++x)
        for (int y = x; y < 3; ++y)
          acc[3 + sym6(x, y)] += t * ((x == y ? S.u : 0.0) + S.du * r[x] * r[y] * is);
      for (int x = 0; x < 3; ++x)
        for (int y = x; y < 3; ++y)
          for (int g = 0; g < 3; ++g)
            acc[9 + 3 * sym6(x, y) + g] +=
                t * (S.dw * r[g] * is * r[x] * r[y] +
                     S.w * ((x == g ? r[y] : 0.0) + (y == g ? r[x] : 0.0)));
      const double hp = S.dw * s * s + 2.0 * S.w * s;
      for (int c = 0; c < 3; ++c) acc[27 + c] += t * hp * r[c] * is;
    }
  }
#pragma unroll
  for (int c = 0; c < 30; ++c) acc[c] = wsum(acc[c]);
  if (lane == 0) {
    double o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (!(xi < kMinOcc)) {
      const double rho = a.rec[(size_t)kPtRec * i];
      double F, dF, ddF;
      const SplineView<double> &E = ci == 0 ? a.emb_mg : a.emb_h;
      const int m = seg_index(rho, E.dx, E.inv_dx, E.n);
      const double pp = fmin(rho - (double)m * E.dx, E.dx);
      const double k[4] = {E.c[m].a, E.c[m].b, E.c[m].c, E.c[m].d};
      cub_vdd(k, pp, F, dF, ddF);
      const double f = xi * ddF;
      o[0] = f;
      double K[9];
      for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) K[3 * x + y] = acc[3 + sym6(x, y)];
      for (int x = 0; x < 3; ++x)
        for (int y = x; y < 3; ++y) {
          double v = f * acc[x] * acc[y] - acc[27 + x] * acc[27 + y] / 3.0;
          for (int z = 0; z < 3; ++z) v += K[3 * z + x] * K[3 * z + y];
          for (int e = 0; e < 6; ++e)
            v += (e < 3 ? 1.0 : 2.0) * acc[9 + 3 * e + x] * acc[9 + 3 * e + y];
          o[1 + sym6(x, y)] = v;
        }
    }
    double4 *d = reinterpret_cast<double4 *>(hrec + 8 * (size_t)i);
    d[0] = make_double4(o[0], o[1], o[2], o[3]);
    d[1] = make_double4(o[4], o[5], o[6], o[7]);
  }
}

// Pass 2b: H_u (9 per real site) = the self products + the neighbours'
// linear terms of both kinds.
// PAIRS: H_u holds the i = u block only and slot9[9p..] the block of
// neighbour j's terms for every entry p of u's list (0 for an empty j):
// evaluate_D2V_i_Dq2_u_MgHx at (u, u) and (u, j).
template <bool PAIRS>
__global__ void __launch_bounds__(128) pt_hess_kernel(PtArgs a, const double *hrec, double *H,
                                                      double *slot9) {
  const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= a.n_real) return;
  const double xu = a.xb[u].x;
  const int cu = a.code[u];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (PAIRS && xu < kMinOcc)
    for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32)
      for (int c = 0; c < 9; ++c) slot9[9 * (size_t)p + c] = 0.0;
  if (!(xu < kMinOcc)) {
    double mu_[kPtRec];
    ld_rec(a.rec + (size_t)kPtRec * u, mu_);
    const double4 qu = a.pos[u];
    for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32) {
      const int j = a.idx[p];
      const double xj = a.xb[j].x;
      if (PAIRS && xj < kMinOcc)
        for (int c = 0; c < 9; ++c) slot9[9 * (size_t)p + c] = 0.0;
      if (xj < kMinOcc) continue;
      const double4 qj = a.pos[j];
      const int cj = a.code[j], pk = pair_kind(cu, cj), o = a.owner[j];
      const double r[3] = {qj.x - qu.x, qj.y - qu.y, qj.z - qu.z};
      const double rn[3] = {-r[0], -r[1], -r[2]};
      const double s = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const PtSpl S = pt_splines(a.T, pk, cu, cj, s);
      const double t = xu * xj;
      // V_u's terms: embedding and pair radial parts, then the moment parts
      pt_hess_linear(mu_, r, S, t, mu_[1] * xj * S.ddrn + 0.5 * t * S.ddph,
                     mu_[1] * xj * S.drn + 0.5 * t * S.dph, acc);
      // V_j's terms (j's owner record)
      double mo[kPtRec];
      ld_rec(a.rec + (size_t)kPtRec * o, mo);
      const double fj = hrec[8 * (size_t)o];
      if (PAIRS) {
        double hj[6] = {0, 0, 0, 0, 0, 0};
        pt_hess_linear(mo, rn, S, t,
                       fj * (xu * S.drc) * (xu * S.drc) + mo[1] * xu * S.ddrc + 0.5 * t * S.ddph,
                       mo[1] * xu * S.drc + 0.5 * t * S.dph, hj);
        for (int x = 0; x < 3; ++x)
          for (int y = 0; y < 3; ++y) slot9[9 * (size_t)p + 3 * x + y] = hj[sym6(x, y)];
      } else {
        pt_hess_linear(mo, rn, S, t,
                       fj * (xu * S.drc) * (xu * S.drc) + mo[1] * xu * S.ddrc + 0.5 * t * S.ddph,
                       mo[1] * xu * S.drc + 0.5 * t * S.dph, acc);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = wsum(acc[c]);
  if (lane == 0) {
    double h[6];
    for (int c = 0; c < 6; ++c) h[c] = (xu < kMinOcc) ? 0.0 : acc[c] + hrec[8 * (size_t)u + 1 + c];
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) H[9 * (size_t)u + 3 * x + y] = h[sym6(x, y)];
  }
}

// Totals in a fixed order: block b sums a contiguous chunk of sites, the
// final warp sums the blocks' partials.
__global__ void __launch_bounds__(256) pt_totals_part_kernel(int n, const double *V,
                                                             const double *Fq, const double *W,
                                                             double *part) {
  __shared__ double sh[kPtTot][256];
  const int b = blockIdx.x, t = threadIdx.x;
  const int chunk = (n + kPtParts - 1) / kPtParts, lo = b * chunk;
  const int hi = lo + chunk < n ? lo + chunk : n;
  double v[kPtTot];
#pragma unroll
  for (int c = 0; c < kPtTot; ++c) v[c] = 0.0;
  for (int i = lo + t; i < hi; i += 256) {
    if (V) v[0] += V[i];
    if (Fq)
      v[1] += Fq[3 * (size_t)i] * Fq[3 * (size_t)i] +
              Fq[3 * (size_t)i + 1] * Fq[3 * (size_t)i + 1] +
              Fq[3 * (size_t)i + 2] * Fq[3 * (size_t)i + 2];
    for (int c = 0; c < 9; ++c) v[2 + c] += W[9 * (size_t)i + c];
  }
  for (int c = 0; c < kPtTot; ++c) sh[c][t] = v[c];
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h)
      for (int c = 0; c < kPtTot; ++c) sh[c][t] += sh[c][t + h];
    __syncthreads();
  }
  if (t < kPtTot) part[(size_t)b * kPtTot + t] = sh[t][0];
}

__global__ void __launch_bounds__(32) pt_totals_final_kernel(const double *part, double *out) {
  const int lane = threadIdx.x;
  for (int c = 0; c < kPtTot; ++c) {
    double v = 0.0;
    for (int b = lane; b < kPtParts; b += 32) v += part[(size_t)b * kPtTot + c];
    v = wsum(v);
    if (lane == 0) out[c] = v;
  }
}

// q <- diag(F) q0 on the real sites (sigma kept).
__global__ void stretch_kernel(int n, const double4 *q0, double F0, double F1, double F2,
                               double4 *pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 a = q0[i];
  pos[i] = make_double4(F0 * a.x, F1 * a.y, F2 * a.z, pos[i].w);
}

inline int nblk(long long n, int per) { return (int)((n + per - 1) / per); }

}  // namespace
}  // namespace btam

namespace {

// Layout of the system's point-form buffer (doubles): rec (16 n), rho (n),
// V (n), Fq (3 n), W (9 n), partials (64 x 12), totals (12), Hessian
// records (8 n), Hessian blocks (9 n).
struct PtLayout {
  double *rec, *rho, *V, *Fq, *W, *part, *tot, *hrec, *H;
};

int pt_buffers(btam_system *s, PtLayout &L) {
  const int n = s->n_real;
  // the Hessian records start on a 32-byte boundary (double4 stores)
  const size_t hoff = ((size_t)(kPtRec + 14) * n + (size_t)kPtParts * kPtTot + kPtTot + 3) &
                      ~(size_t)3;
  const size_t need = hoff + 17 * (size_t)n;
  if (!s->pt || s->pt_cap < need) {
    BTAM_TRY(dalloc(s->pt, s->st, need));
    s->pt_cap = need;
  }
  double *b = s->pt;
  L.rec = b;
  L.rho = L.rec + (size_t)kPtRec * n;
  L.V = L.rho + n;
  L.Fq = L.V + n;
  L.W = L.Fq + 3 * (size_t)n;
  L.part = L.W + 9 * (size_t)n;
  L.tot = L.part + (size_t)kPtParts * kPtTot;
  L.hrec = b + hoff;
  L.H = L.hrec + 8 * (size_t)n;
  return BTAM_OK;
}

PtArgs pt_args(btam_system *s, const PtLayout &L);

// Enqueues both passes and the totals on the system's stream.
int pt_run(btam_system *s, const PtLayout &L) {
  const PtArgs a = pt_args(s, L);
  const int g = nblk((long long)s->n_real * 32, 128);
  pt_moments_kernel<<<g, 128, 0, s->st>>>(a);
  pt_grad_kernel<false><<<g, 128, 0, s->st>>>(a, nullptr);
  pt_totals_part_kernel<<<kPtParts, 256, 0, s->st>>>(s->n_real, L.V, L.Fq, L.W, L.part);
  pt_totals_final_kernel<<<1, 32, 0, s->st>>>(L.part, L.tot);
  return cuda_status(cudaGetLastError());
}

PtArgs pt_args(btam_system *s, const PtLayout &L) {
  PtArgs a;
  a.n_real = s->n_real;
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.owner = s->owner;
  a.offs = s->offs;
  a.idx = s->idx;
  a.T = s->T->r64;
  a.emb_mg = s->T->v64.t[T_F_MG];
  a.emb_h = s->T->v64.t[T_F_H];
  a.rec = L.rec;
  a.rho = L.rho;
  a.V = L.V;
  a.Fq = L.Fq;
  a.W = L.W;
  return a;
}

}  // namespace

// The point-form buffer's W, partials and totals, for the mean-field
// stress (btam_mf_stress), and the fixed-order totals over its sites.
int pt_stress_buffers(btam_system *s, double **W, double **part, double **tot) {
  PtLayout L;
  int st = pt_buffers(s, L);
  if (st != BTAM_OK) return st;
  *W = L.W;
  *part = L.part;
  *tot = L.tot;
  return BTAM_OK;
}
cudaError_t launch_pt_totals(int n, const double *V, const double *Fq, const double *W,
                             double *part, double *tot, cudaStream_t st) {
  pt_totals_part_kernel<<<kPtParts, 256, 0, st>>>(n, V, Fq, W, part);
  pt_totals_final_kernel<<<1, 32, 0, st>>>(part, tot);
  return cudaGetLastError();
}

namespace {

double cell_volume(const GhostBox &b) {
  const double(*A)[3] = b.A;
  return std::fabs(A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                   A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                   A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]));
}

// The cell and origin of a box with every component a scaled by F[a].
void stretched_cell(const GhostBox &b, const double F[3], double origin[3], double cell[9]) {
  for (int a = 0; a < 3; ++a) {
    origin[a] = F[a] * b.origin[a];
    for (int r = 0; r < 3; ++r) cell[3 * r + a] = F[a] * b.A[r][a];
  }
}

// Sets q = diag(F) q0 on the real sites and moves the images with a box
// stretched by F (image = owner + integer combination of the cell rows).
int apply_stretch(btam_system *s, const double4 *q0, const GhostBox &box0, const double F[3],
                  GhostBox &boxF) {
  boxF = box0;
  for (int r = 0; r < 3; ++r)
    for (int a = 0; a < 3; ++a) boxF.A[r][a] = F[a] * box0.A[r][a];
  if (s->n_real > 0)
    stretch_kernel<<<nblk(s->n_real, 256), 256, 0, s->st>>>(s->n_real, q0, F[0], F[1], F[2],
                                                            s->pos);
  BTAM_TRY(cudaGetLastError());
  if (s->n_ghost > 0)
    BTAM_TRY(launch_ghost_refresh(s->n_real, s->n_ghost, s->pos, s->xb, s->code, s->owner,
                                  s->image, boxF, s->st));
  return BTAM_OK;
}

// 3x3 solve by Gaussian elimination with partial pivoting; false if singular.
bool solve3(double J[3][3], double b[3], double x[3]) {
  int p[3] = {0, 1, 2};
  for (int c = 0; c < 3; ++c) {
    int best = c;
    for (int r = c + 1; r < 3; ++r)
      if (std::fabs(J[p[r]][c]) > std::fabs(J[p[best]][c])) best = r;
    std::swap(p[c], p[best]);
    const double d = J[p[c]][c];
    if (!(std::fabs(d) > 0.0) || !std::isfinite(d)) return false;
    for (int r = c + 1; r < 3; ++r) {
      const double f = J[p[r]][c] / d;
      for (int k = c; k < 3; ++k) J[p[r]][k] -= f * J[p[c]][k];
      b[p[r]] -= f * b[p[c]];
    }
  }
  for (int c = 2; c >= 0; --c) {
    double v = b[p[c]];
    for (int k = c + 1; k < 3; ++k) v -= J[p[c]][k] * x[k];
    x[c] = v / J[p[c]][c];
  }
  return std::isfinite(x[0]) && std::isfinite(x[1]) && std::isfinite(x[2]);
}

double norm3(const double y[3]) { return std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]); }

}  // namespace

extern "C" {

int btam_pt_eval(btam_system *s, double *rho, double *V, double *Fq, double *W,
                 double *totals) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  PtLayout L;
  int st = pt_buffers(s, L);
  if (st != BTAM_OK) return st;
  if ((st = pt_run(s, L)) != BTAM_OK) return st;
  const size_t n = (size_t)s->n_real;
  if (rho) BTAM_TRY(cudaMemcpyAsync(rho, L.rho, n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (V) BTAM_TRY(cudaMemcpyAsync(V, L.V, n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (Fq) BTAM_TRY(cudaMemcpyAsync(Fq, L.Fq, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (W) BTAM_TRY(cudaMemcpyAsync(W, L.W, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (totals)
    BTAM_TRY(cudaMemcpyAsync(totals, L.tot, kPtTot * sizeof(double), cudaMemcpyDeviceToHost,
                             s->st));
  return read_err(s);
}

int btam_pt_hessian(btam_system *s, double *H) {
  if (!s || !H) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  PtLayout L;
  int st = pt_buffers(s, L);
  if (st != BTAM_OK) return st;
  const PtArgs a = pt_args(s, L);
  const int g = nblk((long long)s->n_real * 32, 128);
  pt_moments_kernel<<<g, 128, 0, s->st>>>(a);
  pt_hself_kernel<<<g, 128, 0, s->st>>>(a, L.hrec);
  pt_hess_kernel<false><<<g, 128, 0, s->st>>>(a, L.hrec, L.H, nullptr);
  BTAM_TRY(cudaGetLastError());
  BTAM_TRY(cudaMemcpyAsync(H, L.H, 9 * (size_t)s->n_real * sizeof(double),
                           cudaMemcpyDeviceToHost, s->st));
  return read_err(s);
}

int btam_pt_pair_terms(btam_system *s, double *self3, double *slot3, double *Hself,
                       double *Hslot, long long slot_cap) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  int n_slots = 0;
  BTAM_TRY(copy_sync(&n_slots, s->offs + s->n_real, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  if ((slot3 || Hslot) && slot_cap < n_slots) return BTAM_ERR_ARG;
  PtLayout L;
  int st = pt_buffers(s, L);
  if (st != BTAM_OK) return st;
  const size_t n = (size_t)s->n_real;
  double *d_slot = nullptr;
  BTAM_TRY(dalloc(d_slot, s->st, 9 * (size_t)n_slots));
  const PtArgs a = pt_args(s, L);
  const int g = nblk((long long)s->n_real * 32, 128);
  pt_moments_kernel<<<g, 128, 0, s->st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && (self3 || slot3)) {
    pt_grad_kernel<true><<<g, 128, 0, s->st>>>(a, d_slot);
    e = cudaGetLastError();
    if (e == cudaSuccess && self3)
      e = cudaMemcpyAsync(self3, L.Fq, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess && slot3)
      e = cudaMemcpyAsync(slot3, d_slot, 3 * (size_t)n_slots * sizeof(double),
                          cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);  // d_slot is reused below
  }
  if (e == cudaSuccess && (Hself || Hslot)) {
    pt_hself_kernel<<<g, 128, 0, s->st>>>(a, L.hrec);
    pt_hess_kernel<true><<<g, 128, 0, s->st>>>(a, L.hrec, L.H, d_slot);
    e = cudaGetLastError();
    if (e == cudaSuccess && Hself)
      e = cudaMemcpyAsync(Hself, L.H, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess && Hslot)
      e = cudaMemcpyAsync(Hslot, d_slot, 9 * (size_t)n_slots * sizeof(double),
                          cudaMemcpyDeviceToHost, s->st);
  }
  dfree(d_slot, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  return read_err(s);
}

int btam_stretch_apply(btam_system *s, const double F[3]) {
  if (!s || !F) return BTAM_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    if (!(std::isfinite(F[a]) && F[a] > 0.0)) return BTAM_ERR_ARG;
  double origin[3], cell[9];
  stretched_cell(s->box, F, origin, cell);
  GhostBox nb;
  int st = make_box_for(origin, cell, s->box.periodic, nb);
  if (st != BTAM_OK) return st;
  double4 *q0 = nullptr;
  BTAM_TRY(dalloc(q0, s->st, s->n_real));
  cudaError_t e = cudaMemcpyAsync(q0, s->pos, (size_t)s->n_real * sizeof(double4),
                                  cudaMemcpyDeviceToDevice, s->st);
  GhostBox tmp;
  if (e == cudaSuccess) st = apply_stretch(s, q0, s->box, F, tmp);
  dfree(q0, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  if (st != BTAM_OK) return st;
  s->box = nb;
  return read_err(s);
}

}  // extern "C"

namespace {


// form 0: the non-mean-field stress (the reference's bulk residual);
// 1, 2: the mean-field stress at fixed sigma and x, FP64 or FP32C.
// method 0: Newton with a forward-difference Jacobian and backtracking;
// 1: N-GMRES(m) with the critical-point line search (ngmres_stretch).
int relax_stretch(btam_system *s, int form, double atol, double rtol, int max_iter,
                  double F[3], double *info, int method = 0, int m = 3) {
  if (!s || !F || !(atol >= 0.0) || !(rtol >= 0.0) || max_iter < 0) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  for (int a = 0; a < 3; ++a)
    if (!(std::isfinite(F[a]) && F[a] > 0.0)) return BTAM_ERR_ARG;
  const double vol = cell_volume(s->box);
  if (!(vol > 0.0)) return BTAM_ERR_ARG;
  PtLayout L;
  int st = pt_buffers(s, L);
  if (st != BTAM_OK) return st;
  double4 *q0 = nullptr;
  BTAM_TRY(dalloc(q0, s->st, s->n_real));
  BTAM_TRY(cudaMemcpyAsync(q0, s->pos, (size_t)s->n_real * sizeof(double4),
                           cudaMemcpyDeviceToDevice, s->st));
  const GhostBox box0 = s->box;
  int evals = 0;
  // Y_a(X) = (1/V0) sum_u dV_u/dF(a, a) at q = diag(F) q0, F_aa = X_a when
  // X_a > 0 (Mechanical-Relaxation-bulk.cpp:505-511, 570-584)
  auto residual = [&](const double X[3], double Y[3]) -> int {
    double Fx[3];
    for (int a = 0; a < 3; ++a) Fx[a] = X[a] > 0.0 ? X[a] : 1.0;
    GhostBox bF;
    int r = apply_stretch(s, q0, box0, Fx, bF);
    double *dtot = L.tot;
    if (r == BTAM_OK) {
      if (form == 0) {
        r = pt_run(s, L);
      } else {
        double *W = nullptr;
        r = mf_stress_enqueue(s, form == 1 ? BTAM_FP64 : BTAM_FP32C, &W, &dtot);
      }
    }
    double tot[kPtTot];
    if (r == BTAM_OK)
      r = cuda_status(cudaMemcpyAsync(tot, dtot, sizeof(tot), cudaMemcpyDeviceToHost, s->st));
    if (r == BTAM_OK) r = read_err(s);
    if (r != BTAM_OK) return r;
    ++evals;
    // W is taken at q0 = q; the reference's dV/dF(a, a) at the unstretched
    // q0 is W(a, a) / F_aa
    for (int a = 0; a < 3; ++a) Y[a] = tot[2 + 4 * a] / (Fx[a] * vol);
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(Y[a])) return BTAM_ERR_NONFINITE;
    return BTAM_OK;
  };
  double X[3] = {F[0], F[1], F[2]}, Y[3];
  int status = 0, it = 0;
  st = residual(X, Y);
  const double n0 = norm3(Y);
  double nY = n0;
  if (st == BTAM_OK && method == 1) {
    if (nY <= atol || nY <= rtol * n0) status = 1;
    else st = btam::ngmres_stretch(residual, m, atol, rtol, max_iter, X, Y, n0, it, status);
    nY = norm3(Y);
  }
  while (st == BTAM_OK && method == 0) {
    if (nY <= atol || nY <= rtol * n0) {
      status = 1;
      break;
    }
    if (it >= max_iter) break;
    // Jacobian by forward differences, one column per evaluation (the
    // reference's MatFDColoring of a dense 3x3 pattern: three colours,
    // step sqrt(eps) |X_a|, at least 1e-6 sqrt(eps)); the FP32C stress
    // carries ~1e-7 relative noise, so its step is 1e-4 |X_a|
    const double hrel = form == 2 ? 1e-4 : 1.4901161193847656e-08;
    double J[3][3];
    for (int c = 0; c < 3 && st == BTAM_OK; ++c) {
      double Xp[3] = {X[0], X[1], X[2]}, Yp[3];
      double h = hrel * std::fabs(X[c]);
      if (h < 1e-6 * hrel) h = 1e-6 * hrel;
      Xp[c] += h;
      h = Xp[c] - X[c];
      st = residual(Xp, Yp);
      for (int r = 0; r < 3; ++r) J[r][c] = (Yp[r] - Y[r]) / h;
    }
    if (st != BTAM_OK) break;
    double d[3], rhs[3] = {-Y[0], -Y[1], -Y[2]};
    if (!solve3(J, rhs, d)) {
      status = -1;
      break;
    }
    // backtracking on |Y|^2 / 2 along the Newton direction (slope -|Y|^2)
    bool ok = false;
    double lam = 1.0, Xn[3], Yn[3];
    for (int ls = 0; ls < 40 && st == BTAM_OK; ++ls) {
      for (int a = 0; a < 3; ++a) Xn[a] = X[a] + lam * d[a];
      st = residual(Xn, Yn);
      if (st != BTAM_OK) break;
      const double f0 = 0.5 * nY * nY, f1 = 0.5 * norm3(Yn) * norm3(Yn);
      if (f1 <= f0 - 1e-4 * lam * nY * nY) {
        ok = true;
        break;
      }
      lam *= 0.5;
    }
    if (st != BTAM_OK) break;
    if (!ok) {
      status = -1;
      break;
    }
    for (int a = 0; a < 3; ++a) {
      X[a] = Xn[a];
      Y[a] = Yn[a];
    }
    nY = norm3(Y);
    ++it;
  }
  if (st == BTAM_OK) {
    // leave the system stretched by the final F, its cell and origin too
    // (Mechanical-Relaxation-bulk.cpp:366-384)
    double Fx[3];
    for (int a = 0; a < 3; ++a) Fx[a] = X[a] > 0.0 ? X[a] : 1.0;
    double origin[3], cell[9];
    stretched_cell(box0, Fx, origin, cell);
    GhostBox nb;
    st = make_box_for(origin, cell, box0.periodic, nb);
    if (st == BTAM_OK) {
      GhostBox tmp;
      st = apply_stretch(s, q0, box0, Fx, tmp);
      if (st == BTAM_OK) s->box = nb;
    } else {
      GhostBox tmp;  // the stretched cell is too small for its images: undo
      const double one[3] = {1.0, 1.0, 1.0};
      apply_stretch(s, q0, box0, one, tmp);
    }
    for (int a = 0; a < 3; ++a) F[a] = Fx[a];
  }
  dfree(q0, s->st);
  if (st == BTAM_OK) st = read_err(s);
  if (info) {
    info[0] = nY;
    info[1] = it;
    info[2] = evals;
    info[3] = status;
    info[4] = vol;
  }
  return st;
}

}  // namespace

extern "C" {

int btam_relax_stretch(btam_system *s, double atol, double rtol, int max_iter, double F[3],
                       double *info) {
  return relax_stretch(s, 0, atol, rtol, max_iter, F, info);
}

int btam_relax_stretch_ngmres(btam_system *s, int m, double atol, double rtol, int max_iter,
                              double F[3], double *info) {
  if (m < 1) return BTAM_ERR_ARG;
  return relax_stretch(s, 0, atol, rtol, max_iter, F, info, 1, m);
}

int btam_relax_stretch_mf(btam_system *s, int precision, double atol, double rtol,
                          int max_iter, double F[3], double *info) {
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  return relax_stretch(s, precision == BTAM_FP64 ? 1 : 2, atol, rtol, max_iter, F, info);
}

}  // extern "C"
