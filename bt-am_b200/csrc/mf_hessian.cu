// Mean-field Hessian blocks: evaluate_D2V0_i_Dmeanq2_u_MgHx
// (MgHx-mf-V-bulk.cpp:1366-1600) summed over i in {u} U N(u), on the
// device.  No solver here or in the reference calls it (the Newton option
// of the relaxation is matrix-free); it serves the plugin table's last slot
// and callers that want a block preconditioner.  So the kernel evaluates
// the reference's sums directly, term by term at the rule's points, instead
// of through the moment decomposition of the hot path:
//   i = u: the pair terms (12 points) and every triplet (u, j1, j2),
//          j1 <= j2 in u's list (18 points, 12 for j1 = j2), block (0, 0)
//          of each term's Hessian, averaged over the points;
//   i a neighbour of u (real or periodic image, whose terms are its owner's
//          translated): the pair (i, u) and the triplets of i's list that
//          hold u, the block of u's slot (for j1 = j2 = u the two slot
//          blocks without their cross blocks, as the reference sums them);
//   plus each i's embedding x_i F''(rho_i) g g^T + x_i F'(rho_i) <d2 rho>,
//   from the pair terms that hold u.
// A warp per real site; lanes over its list entries; FP64; the block sums
// are symmetric, so six entries are reduced.  Per site the work is about
// N_nb^2 x 18 term Hessians (tens of milliseconds for 27,000 sites).
#include <cmath>

#include "internal.cuh"

namespace btam {
namespace {

// Spline value and first and second derivatives of a segment record.
__device__ __forceinline__ void seg_vdd(const double *k, double p, double &v, double &d1,
                                        double &d2) {
  v = k[0] + (k[1] + (k[2] + k[3] * p) * p) * p;
  d1 = k[1] + (2.0 * k[2] + 3.0 * k[3] * p) * p;
  d2 = 2.0 * k[2] + 6.0 * k[3] * p;
}

struct Spl3 {
  double v, d1, d2;
};

__device__ __forceinline__ void uw_at(const RadialView<double> &T, int pk, double s, Spl3 &u,
                                      Spl3 &w) {
  double p;
  const int m = seg_of(T, s, p);
  double k[8];
  ld8(uw_rec(T, pk, m), k);
  seg_vdd(k, p, u.v, u.d1, u.d2);
  seg_vdd(k + 4, p, w.v, w.d1, w.d2);
}

// phi of pair kind pk and rho of species c at s.
__device__ __forceinline__ void pr_at2(const RadialView<double> &T, int pk, int c, double s,
                                       Spl3 &ph, Spl3 &rho) {
  double p;
  const int m = seg_of(T, s, p);
  const double *pr = pr_rec(T, pk, m);
  double k[4];
  for (int q = 0; q < 4; ++q) k[q] = pr[q];
  seg_vdd(k, p, ph.v, ph.d1, ph.d2);
  const int o = rho_off(pk, c);
  for (int q = 0; q < 4; ++q) k[q] = pr[o + q];
  seg_vdd(k, p, rho.v, rho.d1, rho.d2);
}

__device__ __forceinline__ double nrm(const double *r) {
  return sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

// Symmetric 3x3 accumulators as xx yy zz yz xz xy.
__device__ __forceinline__ int s6(int a, int b) {
  return a == b ? a : (a + b == 3 ? 3 : (a + b == 2 ? 4 : 5));
}

// H += c (f'' P + f' Q), P = r r^T / s^2, Q = (I - P) / s.
__device__ __forceinline__ void add_radial(const double *r, double s, double d1, double d2,
                                           double c, double (&H)[6]) {
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      const double P = r[a] * r[b] / (s * s);
      H[s6(a, b)] += c * (d2 * P + d1 * ((a == b ? 1.0 : 0.0) - P) / s);
    }
}

// H += sum_al m_al d2 A_al with A = c u(|r|) r.
__device__ __forceinline__ void add_vec(const double *m, const double *r, double s,
                                        const Spl3 &u, double c, double (&H)[6]) {
  const double mr = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      const double P = r[a] * r[b] / (s * s);
      H[s6(a, b)] += c * (u.d1 * (m[a] * r[b] + r[a] * m[b]) / s +
                          mr * (u.d2 * P + u.d1 * ((a == b ? 1.0 : 0.0) - P) / s));
    }
}

// H += sum_ab M_ab d2 B_ab with B = c w(|r|) r r^T (M symmetric, 3x3 full).
__device__ __forceinline__ void add_ten(const double *M, const double *r, double s,
                                        const Spl3 &w, double c, double (&H)[6]) {
  double Mr[3];
  for (int a = 0; a < 3; ++a) Mr[a] = M[3 * a] * r[0] + M[3 * a + 1] * r[1] + M[3 * a + 2] * r[2];
  const double rMr = r[0] * Mr[0] + r[1] * Mr[1] + r[2] * Mr[2];
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      const double P = r[a] * r[b] / (s * s);
      H[s6(a, b)] += c * (rMr * (w.d2 * P + w.d1 * ((a == b ? 1.0 : 0.0) - P) / s) +
                          2.0 * w.d1 * (r[a] * Mr[b] + Mr[a] * r[b]) / s + 2.0 * w.v * M[3 * a + b]);
    }
}

// Blocks of the triplet terms at one geometry (r_k = q_0 - q_k, c_k = n_0 n_k):
// block 0 (the centre) or block 1 (slot 1 alone) of V_dip + V_quad, times f.
__device__ void triplet_block(int blk, const double *r1, const double *r2, double c1, double c2,
                              const Spl3 &u1, const Spl3 &w1, const Spl3 &u2, const Spl3 &w2,
                              double f, double (&H)[6]) {
  const double s1 = nrm(r1), s2 = nrm(r2);
  double h[6] = {0, 0, 0, 0, 0, 0};
  double A1[3], A2[3], B1[9], B2[9];
  for (int k = 0; k < 3; ++k) {
    A1[k] = c1 * u1.v * r1[k];
    A2[k] = c2 * u2.v * r2[k];
  }
  for (int x = 0; x < 3; ++x)
    for (int y = 0; y < 3; ++y) {
      B1[3 * x + y] = c1 * w1.v * r1[x] * r1[y];
      B2[3 * x + y] = c2 * w2.v * r2[x] * r2[y];
    }
  const double t1 = c1 * w1.v * s1 * s1, t2 = c2 * w2.v * s2 * s2;
  const double hp1 = w1.d1 * s1 * s1 + 2.0 * w1.v * s1;
  const double hpp1 = w1.d2 * s1 * s1 + 4.0 * w1.d1 * s1 + 2.0 * w1.v;
  const double hp2 = w2.d1 * s2 * s2 + 2.0 * w2.v * s2;
  const double hpp2 = w2.d2 * s2 * s2 + 4.0 * w2.d1 * s2 + 2.0 * w2.v;
  // dipole 1/2 A1.A2 and quadrupole 1/2 B1:B2 - t1 t2 / 6: parts linear in
  // the other slot's feature
  add_vec(A2, r1, s1, u1, 0.5 * c1, h);
  add_ten(B2, r1, s1, w1, 0.5 * c1, h);
  add_radial(r1, s1, hp1, hpp1, -t2 * c1 / 6.0, h);
  if (blk == 0) {
    add_vec(A1, r2, s2, u2, 0.5 * c2, h);
    add_ten(B1, r2, s2, w2, 0.5 * c2, h);
    add_radial(r2, s2, hp2, hpp2, -t1 * c2 / 6.0, h);
    // cross parts: J1^T J2 + J2^T J1 (dipole), dB1:dB2 sym (quadrupole),
    // grad t1 grad t2^T sym (trace)
    const double d12 = r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2];
    for (int x = 0; x < 3; ++x)
      for (int y = x; y < 3; ++y) {
        double jj = 0.0;
        for (int z = 0; z < 3; ++z) {
          const double J1zx = c1 * ((z == x ? u1.v : 0.0) + u1.d1 * r1[z] * r1[x] / s1);
          const double J1zy = c1 * ((z == y ? u1.v : 0.0) + u1.d1 * r1[z] * r1[y] / s1);
          const double J2zx = c2 * ((z == x ? u2.v : 0.0) + u2.d1 * r2[z] * r2[x] / s2);
          const double J2zy = c2 * ((z == y ? u2.v : 0.0) + u2.d1 * r2[z] * r2[y] / s2);
          jj += J1zx * J2zy + J2zx * J1zy;
        }
        auto G = [&](int p, int q) {
          return c1 * c2 *
                 (w1.d1 * w2.d1 * (r1[p] / s1) * (r2[q] / s2) * d12 * d12 +
                  2.0 * w1.d1 * w2.v * (r1[p] / s1) * r1[q] * d12 +
                  2.0 * w1.v * w2.d1 * r2[p] * (r2[q] / s2) * d12 +
                  2.0 * w1.v * w2.v * ((p == q ? d12 : 0.0) + r2[p] * r1[q]));
        };
        const double g1x = c1 * hp1 * r1[x] / s1, g1y = c1 * hp1 * r1[y] / s1;
        const double g2x = c2 * hp2 * r2[x] / s2, g2y = c2 * hp2 * r2[y] / s2;
        h[s6(x, y)] += 0.5 * jj + 0.5 * (G(x, y) + G(y, x)) - (g1x * g2y + g2x * g1y) / 6.0;
      }
  }
  for (int c = 0; c < 6; ++c) H[c] += f * h[c];
}

struct MfhArgs {
  int n_real;
  const double4 *pos;  // q, sigma
  const double2 *xb;
  const int *code, *owner, *offs, *idx;
  const double *rho;  // mean-field rho-bar of the real sites
  // null: the rho gradients come from the degree-3 rule's points; else, per
  // list entry p of a real site i, the gradient of rho_ij (j = idx[p]) in
  // q_i that replaces them (the multipole rule's, whose gradient in q_j is
  // its exact negative)
  const double *gmp;
  RadialView<double> T;
  SplineView<double> emb_mg, emb_h;
  double *H;
  // null: H sums over i in {u} U N(u); else H holds the i = u block only and
  // Hslot (9 per entry p of the real sites' lists) the block of neighbour
  // idx[p]: the reference's per-pair values
  double *Hslot = nullptr;
};

__device__ __forceinline__ bool skipped(const MfhArgs &a, int j) {
  const double x = a.xb[j].x;
  return a.code[j] == 1 && x <= kMinOcc;  // H neighbours at or below min_occupancy
}

// Adds the rule-averaged blocks of the pair (c, nb) terms for the slot
// `blk` (0: the centre, 1: the neighbour) and the rho gradient of that slot.
__device__ void pair_terms(const MfhArgs &a, const double *rc, int cc, double xc, double sc,
                           const double *rn, int cn, double xn, double sn, int blk, double *g,
                           double (&d2rho)[6], double (&pair)[6]) {
  const int pk = pair_kind(cc, cn);
  for (int l = 0; l < 6; ++l)
    for (int sg = 0; sg < 2; ++sg) {
      double r[3] = {rc[0] - rn[0], rc[1] - rn[1], rc[2] - rn[2]};
      const double amt = (sg ? -1.0 : 1.0) * kDelta6 * (l < 3 ? sc : sn);
      r[l % 3] += l < 3 ? amt : -amt;
      const double s = nrm(r);
      Spl3 ph, rh;
      pr_at2(a.T, pk, cn, s, ph, rh);
      for (int k = 0; k < 3; ++k) g[k] += kW6 * (blk == 0 ? 1.0 : -1.0) * xn * rh.d1 * r[k] / s;
      add_radial(r, s, rh.d1, rh.d2, kW6 * xn, d2rho);
      add_radial(r, s, ph.d1, ph.d2, kW6 * 0.5 * xc * xn, pair);
    }
}

// Adds the rule-averaged triplet block: centre c, slots j1 (relative r1 =
// q_c - q_j1) and j2; coincident j1 = j2 uses the merged 12-point measure
// and (for blk 1) both slot blocks.
__device__ void triplet_terms(const MfhArgs &a, const double *r1_0, const double *r2_0, int cc,
                              double xc, double sc, int c1s, double x1, double s1s, int c2s,
                              double x2, double s2s, bool coincident, int blk, double f,
                              double (&H)[6]) {
  const int pk1 = pair_kind(cc, c1s), pk2 = pair_kind(cc, c2s);
  const double cf1 = xc * x1, cf2 = xc * x2;
  const int D = coincident ? 6 : 9;
  const double delta = coincident ? kDelta6 : kDelta9, W = coincident ? kW6 : kW9;
  for (int l = 0; l < D; ++l)
    for (int sg = 0; sg < 2; ++sg) {
      double r1[3] = {r1_0[0], r1_0[1], r1_0[2]}, r2[3] = {r2_0[0], r2_0[1], r2_0[2]};
      const double sgn = sg ? -1.0 : 1.0;
      const int ax = l % 3, grp = l / 3;  // 0: centre, 1: j1 (both slots when coincident), 2: j2
      if (grp == 0) {
        r1[ax] += sgn * delta * sc;
        r2[ax] += sgn * delta * sc;
      } else if (grp == 1) {
        r1[ax] -= sgn * delta * s1s;
        if (coincident) r2[ax] -= sgn * delta * s1s;
      } else {
        r2[ax] -= sgn * delta * s2s;
      }
      Spl3 u1, w1, u2, w2;
      uw_at(a.T, pk1, nrm(r1), u1, w1);
      uw_at(a.T, pk2, nrm(r2), u2, w2);
      if (blk == 0) {
        triplet_block(0, r1, r2, cf1, cf2, u1, w1, u2, w2, f * W, H);
      } else {
        triplet_block(1, r1, r2, cf1, cf2, u1, w1, u2, w2, f * W, H);
        if (coincident) triplet_block(1, r2, r1, cf2, cf1, u2, w2, u1, w1, f * W, H);
      }
    }
}

__device__ __forceinline__ void emb_dd(const SplineView<double> &E, double rho, double &d1,
                                       double &d2) {
  const int m = seg_index(rho, E.dx, E.inv_dx, E.n);
  const double p = fmin(rho - (double)m * E.dx, E.dx);
  const double k[4] = {E.c[m].a, E.c[m].b, E.c[m].c, E.c[m].d};
  double v;
  seg_vdd(k, p, v, d1, d2);
}

__global__ void __launch_bounds__(128) mf_hess_kernel(MfhArgs a) {
  const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= a.n_real) return;
  const double4 pu = a.pos[u];
  const double xu = a.xb[u].x;
  const int cu = a.code[u];
  const bool live = !(cu == 1 && xu < kMinOcc);  // 1398-1402
  const double qu[3] = {pu.x, pu.y, pu.z};
  double hs[6] = {0, 0, 0, 0, 0, 0};       // i = u: pair, triplet and x F' d2rho parts
  double gsum[3] = {0, 0, 0}, d2s[6] = {0, 0, 0, 0, 0, 0};
  double hn[6] = {0, 0, 0, 0, 0, 0};       // i = neighbours: everything
  const int nb0 = a.offs[u], nb1 = a.offs[u + 1];
  if (a.Hslot)
    for (int k1 = nb0 + lane; k1 < nb1; k1 += 32)
      for (int c = 0; c < 9; ++c) a.Hslot[9 * (size_t)k1 + c] = 0.0;
  if (live) {
    for (int k1 = nb0 + lane; k1 < nb1; k1 += 32) {
      const int j1 = a.idx[k1];
      if (skipped(a, j1)) continue;
      const double4 p1 = a.pos[j1];
      const double q1[3] = {p1.x, p1.y, p1.z};
      const double x1 = a.xb[j1].x;
      const int c1 = a.code[j1];
      // ---- i = u: pair (u, j1), centre block
      double pair[6] = {0, 0, 0, 0, 0, 0};
      double gdeg3[3] = {0, 0, 0};
      pair_terms(a, qu, cu, xu, pu.w, q1, c1, x1, p1.w, 0, a.gmp ? gdeg3 : gsum, d2s, pair);
      if (a.gmp)
        for (int c = 0; c < 3; ++c) gsum[c] += a.gmp[3 * (size_t)k1 + c];
      for (int c = 0; c < 6; ++c) hs[c] += pair[c];
      // triplets (u, j1, j2), j2 at or after j1 in u's list
      const double r1[3] = {qu[0] - q1[0], qu[1] - q1[1], qu[2] - q1[2]};
      for (int k2 = k1; k2 < nb1; ++k2) {
        const int j2 = a.idx[k2];
        if (skipped(a, j2)) continue;
        const double4 p2 = a.pos[j2];
        const double r2[3] = {qu[0] - p2.x, qu[1] - p2.y, qu[2] - p2.z};
        triplet_terms(a, r1, r2, cu, xu, pu.w, c1, x1, p1.w, a.code[j2], a.xb[j2].x, p2.w,
                      k2 == k1, 0, k2 == k1 ? 1.0 : 2.0, hs);
      }
      // ---- i = j1 (its owner's list, translated): the terms that hold u
      if (c1 == 1 && x1 < kMinOcc) continue;  // 1424-1427
      const int o = a.owner[j1];
      const double4 po = a.pos[o];
      const double d[3] = {qu[0] - q1[0], qu[1] - q1[1], qu[2] - q1[2]};  // u seen from j1
      int ks = -1;
      for (int k = a.offs[o]; k < a.offs[o + 1]; ++k) {
        const int j = a.idx[k];
        if (a.owner[j] != u) continue;
        const double4 pj = a.pos[j];
        if (fabs(pj.x - po.x - d[0]) < 1e-8 && fabs(pj.y - po.y - d[1]) < 1e-8 &&
            fabs(pj.z - po.z - d[2]) < 1e-8) {
          ks = k;
          break;
        }
      }
      if (ks < 0) continue;  // u lies outside j1's cutoff sphere
      if (xu <= kMinOcc && cu == 1) continue;
      double gi[3] = {0, 0, 0}, d2i[6] = {0, 0, 0, 0, 0, 0}, hi[6] = {0, 0, 0, 0, 0, 0};
      pair_terms(a, q1, c1, x1, p1.w, qu, cu, xu, pu.w, 1, gi, d2i, hi);
      if (a.gmp)
        for (int c = 0; c < 3; ++c) gi[c] = -a.gmp[3 * (size_t)ks + c];
      const double ru[3] = {-d[0], -d[1], -d[2]};  // q_j1 - q_u
      for (int k2 = a.offs[o]; k2 < a.offs[o + 1]; ++k2) {
        const int j2 = a.idx[k2];
        if (skipped(a, j2)) continue;
        const double4 p2 = a.pos[j2];
        const double r2[3] = {po.x - p2.x, po.y - p2.y, po.z - p2.z};  // q_o - q_j2 = q_j1 - q_j2'
        triplet_terms(a, ru, r2, c1, x1, p1.w, cu, xu, pu.w, a.code[j2], a.xb[j2].x, p2.w,
                      k2 == ks, 1, k2 == ks ? 1.0 : 2.0, hi);
      }
      double dF, ddF;
      emb_dd(c1 == 0 ? a.emb_mg : a.emb_h, a.rho[o], dF, ddF);
      if (a.Hslot) {
        for (int x = 0; x < 3; ++x)
          for (int y = 0; y < 3; ++y) {
            const int c = s6(x < y ? x : y, x < y ? y : x);
            a.Hslot[9 * (size_t)k1 + 3 * x + y] =
                hi[c] + x1 * ddF * gi[x] * gi[y] + x1 * dF * d2i[c];
          }
        continue;
      }
      for (int x = 0; x < 3; ++x)
        for (int y = x; y < 3; ++y)
          hn[s6(x, y)] += hi[s6(x, y)] + x1 * ddF * gi[x] * gi[y] + x1 * dF * d2i[s6(x, y)];
    }
  }
  double out[15];
  for (int c = 0; c < 6; ++c) out[c] = hs[c] + hn[c];
  for (int c = 0; c < 3; ++c) out[6 + c] = gsum[c];
  for (int c = 0; c < 6; ++c) out[9 + c] = d2s[c];
#pragma unroll
  for (int c = 0; c < 15; ++c)
    for (int off = 16; off > 0; off >>= 1) out[c] += __shfl_xor_sync(0xffffffffu, out[c], off);
  if (lane == 0) {
    double h[6] = {0, 0, 0, 0, 0, 0};
    if (live) {
      double dF, ddF;
      emb_dd(cu == 0 ? a.emb_mg : a.emb_h, a.rho[u], dF, ddF);
      for (int x = 0; x < 3; ++x)
        for (int y = x; y < 3; ++y)
          h[s6(x, y)] = out[s6(x, y)] + xu * ddF * out[6 + x] * out[6 + y] +
                        xu * dF * out[9 + s6(x, y)];
    }
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) a.H[9 * (size_t)u + 3 * x + y] = h[s6(x, y)];
  }
}

}  // namespace
}  // namespace btam

int mf_hessian_enqueue(btam_system *s, double *Hd, double *Hslot) {
  int st = mf_rho64_enqueue(s);  // rho-bar of the real sites into the system's rho
  if (st != BTAM_OK) return st;
  return mf_hessian_enqueue_with(s, s->rho, nullptr, Hd, Hslot);
}

int mf_hessian_enqueue_with(btam_system *s, const double *rho, const double *gmp, double *Hd,
                            double *Hslot) {
  MfhArgs a;
  a.n_real = s->n_real;
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.owner = s->owner;
  a.offs = s->offs;
  a.idx = s->idx;
  a.rho = rho;
  a.gmp = gmp;
  a.T = s->T->r64;
  a.emb_mg = s->T->v64.t[T_F_MG];
  a.emb_h = s->T->v64.t[T_F_H];
  a.H = Hd;
  a.Hslot = Hslot;
  const int g = (int)(((long long)s->n_real * 32 + 127) / 128);
  if (g > 0) mf_hess_kernel<<<g, 128, 0, s->st>>>(a);
  return cuda_status(cudaGetLastError());
}

extern "C" {

int btam_mf_hessian(btam_system *s, double *H) {
  if (!s || !H) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  double *Hd = nullptr;
  BTAM_TRY(dalloc(Hd, s->st, 9 * (size_t)s->n_real));
  int st = mf_hessian_enqueue(s, Hd, nullptr);
  if (st != BTAM_OK) {
    dfree(Hd, s->st);
    return st;
  }
  const cudaError_t e = cudaMemcpyAsync(H, Hd, 9 * (size_t)s->n_real * sizeof(double),
                                        cudaMemcpyDeviceToHost, s->st);
  dfree(Hd, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  return read_err(s);
}

int btam_mf_hessian_pairs(btam_system *s, double *Hself, double *Hslot, long long slot_cap) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  int n_slots = 0;
  BTAM_TRY(copy_sync(&n_slots, s->offs + s->n_real, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  if (Hslot && slot_cap < n_slots) return BTAM_ERR_ARG;
  double *Hd = nullptr, *Hs = nullptr;
  BTAM_TRY(dalloc(Hd, s->st, 9 * (size_t)s->n_real));
  cudaError_t e = dalloc(Hs, s->st, 9 * (size_t)n_slots);
  int st = e == cudaSuccess ? mf_hessian_enqueue(s, Hd, Hs) : cuda_status(e);
  if (st == BTAM_OK && Hself)
    st = cuda_status(cudaMemcpyAsync(Hself, Hd, 9 * (size_t)s->n_real * sizeof(double),
                                     cudaMemcpyDeviceToHost, s->st));
  if (st == BTAM_OK && Hslot)
    st = cuda_status(cudaMemcpyAsync(Hslot, Hs, 9 * (size_t)n_slots * sizeof(double),
                                     cudaMemcpyDeviceToHost, s->st));
  dfree(Hd, s->st);
  dfree(Hs, s->st);
  if (st != BTAM_OK) return st;
  return read_err(s);
}

}  // extern "C"
