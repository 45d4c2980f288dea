// Mean-field ADP arithmetic shared by the CUDA kernels (adp_kernels.cu).
//
// The reference evaluates, per site i, the degree-3 Gauss-Hermite average of
// the ADP terms over its neighbours (MgHx-mf-V-bulk.cpp:708-953): the pair
// terms rho and phi with the 12-point pair rule (dimension 6, offset
// sqrt(6) sigma, weight 1/12) and the dipole/quadrupole terms over all
// neighbour pairs j1 <= j2 with the 18-point triplet rule (dimension 9,
// offset 3 sigma, weight 1/18) or, for j1 == j2, the merged 12-point rule.
// Every quadrature point moves exactly one group along one axis, and the
// angular terms are the symmetric bilinear form
//     B(g1, g2) = 1/2 a1.a2 + 1/2 L1:L2 - 1/6 tr L1 tr L2
// of the per-neighbour features g = (a, L) = x_i x_j (u(r) r, w(r) r (x) r)
// (MgHx-ADP.cpp:1233-1281, 1781-1831).  So the O(N_nb^2) triplet sum is
// exactly, up to rounding, a sum of O(N_nb) per-site moments:
//   sum_{j1<=j2} f * <V_ang>  =  1/18 sum_d [B(G(d),G(d)) - sum_j B(g_j(d),g_j(d))]
//                              + 2/18 [B(H, G0) - sum_j B(h_j, g_j(r0))]
//                              + 1/12 sum_j sum_{12 pts} B(g_j, g_j)
// with G0 = sum_j g_j(r0_j), G(d) = sum_j g_j(r0_j + d) for the six centre
// displacements d = +-3 sigma_i e_k, h_j = sum of g_j over the six
// neighbour displacements -+3 sigma_j e_k, H = sum_j h_j.  Gradients are the
// exact derivatives of this closed form, which equals what the reference's
// _dmq/_dsq/_dxi rules return (Quadrature-Hermitian-3th.cpp:114-378).
//
// Pass 1 (per centre site) accumulates rho-bar, the pair/diagonal energies
// and the moments G0, G(d), H; pass 2 (per site u, over its neighbours j)
// adds dV0_u/d(q_u, sigma_u) from u's moments and dV0_j/d(q_u, sigma_u, x_u)
// from j's moments.  All functions here are per pair and templated on the
// arithmetic type R (double: plain FP64 form; float: FP32 form whose callers
// accumulate with compensated sums).
#pragma once

#if defined(__CUDACC__)
#define BTAM_HD __host__ __device__ __forceinline__
#else
#define BTAM_HD inline
#endif

#include <cmath>
#include <cstdint>

namespace btam {

// Degree-3 rule constants (Quadrature-Hermitian-3th.cpp:56-60).
constexpr double kDelta9 = 3.0;                 // sqrt(9)
constexpr double kDelta6 = 2.449489742783178;   // sqrt(6)
constexpr double kW9 = 1.0 / 18.0;
constexpr double kW6 = 1.0 / 12.0;
constexpr double kMinOcc = 5e-4;                // min_occupancy (Macros.hpp:869)

// Table slots in the packed table array.
enum TableId : int {
  T_RHO_MG = 0, T_RHO_H = 1, T_F_MG = 2, T_F_H = 3,
  T_PHI = 4,   // + pair kind (0 MgMg, 1 HH, 2 MgH)
  T_U = 7, T_W = 10, T_COUNT = 13
};

template <class R> struct Coef4 { R a, b, c, d; };

// One uniform-knot cubic spline (cubic-spline.cpp:84-112): segment
// m = min(floor(r/dx), n-1), p = min(r - m dx, dx), value a+(b+(c+d p)p)p,
// derivative b+(2c+3d p)p (the reference's db/dc/dd columns equal b, 2c, 3d).
template <class R> struct SplineView {
  const Coef4<R> *c;
  R dx, inv_dx;
  int n;
};

template <class R> struct TablesView {
  SplineView<R> t[T_COUNT];
};

template <class R> BTAM_HD R rmin(R a, R b) { return a < b ? a : b; }

// Segment index m = min(int(x / dx), n - 1) (cubic-spline.cpp:89-90).  In
// FP64 the index is the reference's: x times 1/dx truncates to the same
// integer as the rounded quotient unless it lies within 1e-9 of a knot, and
// there the quotient itself is taken, so a point on a knot picks the
// reference's segment.  The FP32 form takes the product.  A negative
// argument (an embedding density below 0, which the reference would index
// before its table with) takes segment 0, whose cubic is then extrapolated;
// on the device a NaN argument converts to 0 as well, so no argument reads
// outside the table.
template <class R> BTAM_HD int seg_index(R x, R dx, R inv_dx, int n) {
  const R t = x * inv_dx;
  int m = (int)t;
  if (sizeof(R) == 8) {
    const R f = t - (R)m;
    if (f < (R)1e-9 || f > (R)1 - (R)1e-9) m = (int)(x / dx);
  }
  m = m < n - 1 ? m : n - 1;
  return m > 0 ? m : 0;
}

template <class R>
BTAM_HD void spline_vd(const SplineView<R> &s, R r, R &v, R &dv) {
  const int m = seg_index<R>(r, s.dx, s.inv_dx, s.n);
  R p = rmin(r - (R)m * s.dx, s.dx);
#if defined(__CUDA_ARCH__)
  Coef4<R> k;
  if (sizeof(R) == 4) {
    float4 t = __ldg(reinterpret_cast<const float4 *>(s.c) + m);
    k.a = (R)t.x; k.b = (R)t.y; k.c = (R)t.z; k.d = (R)t.w;
  } else {
    const double2 *q = reinterpret_cast<const double2 *>(s.c) + 2 * m;
    double2 t0 = __ldg(q), t1 = __ldg(q + 1);
    k.a = (R)t0.x; k.b = (R)t0.y; k.c = (R)t1.x; k.d = (R)t1.y;
  }
#else
  Coef4<R> k = s.c[m];
#endif
  v = k.a + (k.b + (k.c + k.d * p) * p) * p;
  dv = k.b + ((R)2 * k.c + (R)3 * k.d * p) * p;
}

template <class R> BTAM_HD R spline_v(const SplineView<R> &s, R r) {
  R v, dv;
  spline_vd(s, r, v, dv);
  return v;
}

// ---------------------------------------------------------------------------
// Kernel form of the radial tables.  Every radial function of the potential
// (rho_Mg, rho_H and phi, u, w of the three pair kinds) is tabulated on one
// uniform knot grid (n = 1194, dx = 0.00527527527528; adpmg.dat:2,
// adph.dat:2, adpmgh.dat:2 and the pair blocks after them), so one segment
// index (m, p) serves every function at a geometry, and the coefficients of
// the functions a geometry needs together sit in one aligned record (one
// 32-byte sector per 8 floats):
//   uw block of pair kind pk (at uw + 8 n pk): 8 R per segment: u (a, b, c,
//           d), w (a, b, c, d);
//   pr block of pair kind pk (at pr + 8 n pk): pr_stride(pk) R per segment:
//           phi (a..d) and rho (a..d) of the species for the same-species
//           kinds; phi, rho_Mg, rho_H and four zeros for Mg-H.
// The blocks are found by arithmetic on the pair kind, not by indexing an
// array of pointers, so lanes of different pair kinds never serialise on a
// divergent parameter-space load.
template <class R> struct RadialView {
  const R *uw;
  const R *pr;
  R dx, inv_dx;
  int n;
  // the uw block again, laid out as the shared-memory kernels stage it
  // (halves swapped where uw_swapped says), for one bulk copy; may be null
  const R *uws = nullptr;
};
constexpr int kUWStride = 8;
BTAM_HD int pr_stride(int pk) { return pk == 2 ? 16 : 8; }
template <class R> BTAM_HD const R *uw_rec(const RadialView<R> &T, int pk, int m) {
  return T.uw + (size_t)kUWStride * ((size_t)T.n * pk + m);
}
// The same tables with the uw block staged in shared memory by the kernel
// (3 pair kinds x n segments x 32 bytes = 115 KB at n = 1194 in FP32,
// x 64 bytes = 229 KB in FP64); the pr block stays in global memory.
template <class R> struct RadialViewS : RadialView<R> {};
template <class R> BTAM_HD const R *pr_rec(const RadialView<R> &T, int pk, int m) {
  return T.pr + (size_t)8 * T.n * pk + (size_t)pr_stride(pk) * m;
}
// Offset of rho of species c (0 Mg, 1 H) in a pr record of pair kind pk.
BTAM_HD int rho_off(int pk, int c) { return (pk == 2 && c == 1) ? 8 : 4; }

// Segment of |r| = s (cubic-spline.cpp:84-96): m = min(floor(s/dx), n-1),
// p = min(s - m dx, dx).
template <class R> BTAM_HD int seg_of(const RadialView<R> &T, R s, R &p) {
  const int m = seg_index<R>(s, T.dx, T.inv_dx, T.n);
  p = rmin(s - (R)m * T.dx, T.dx);
  return m;
}

// Cubic a + (b + (c + d p) p) p and its derivative b + (2c + 3d p) p.
template <class R> BTAM_HD R cub_v(const R *k, R p) {
  return k[0] + (k[1] + (k[2] + k[3] * p) * p) * p;
}
template <class R> BTAM_HD void cub_vd(const R *k, R p, R &v, R &dv) {
  v = cub_v(k, p);
  dv = k[1] + ((R)2 * k[2] + (R)3 * k[3] * p) * p;
}

// Read-only vector loads of 32-byte-aligned records (device: non-coherent
// 256-bit loads; host: plain copies).
BTAM_HD void ld8(const float *p, float (&v)[8]) {
#if defined(__CUDA_ARCH__)
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]),
        "=f"(v[7])
      : "l"(p));
#else
  for (int c = 0; c < 8; ++c) v[c] = p[c];
#endif
}
BTAM_HD void ld8(const double *p, double (&v)[8]) {
#if defined(__CUDA_ARCH__)
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
      : "l"(p));
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(v[4]), "=d"(v[5]), "=d"(v[6]), "=d"(v[7])
      : "l"(p + 4));
#else
  for (int c = 0; c < 8; ++c) v[c] = p[c];
#endif
}
BTAM_HD void ld4(const float *p, float (&v)[4]) {
#if defined(__CUDA_ARCH__)
  float4 t = __ldg(reinterpret_cast<const float4 *>(p));
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
#else
  for (int c = 0; c < 4; ++c) v[c] = p[c];
#endif
}
BTAM_HD void ld4(const double *p, double (&v)[4]) {
#if defined(__CUDA_ARCH__)
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
      : "l"(p));
#else
  for (int c = 0; c < 4; ++c) v[c] = p[c];
#endif
}
// Plain 8-value copy (records staged in shared memory).
template <class R> BTAM_HD void cp8(const R *p, R (&v)[8]) {
  for (int c = 0; c < 8; ++c) v[c] = p[c];
}
// 8 floats of a 32-byte record in shared memory whose two 16-byte halves
// are stored swapped when `swap` (two 128-bit shared loads; host: plain
// copy).  Records stored with their halves swapped on every other group of
// four spread the first loaded halves of random records over all eight
// 16-byte bank groups instead of four.
BTAM_HD void lds8(const float *p, bool swap, float (&v)[8]) {
#if defined(__CUDA_ARCH__)
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  const unsigned a0 = swap ? a + 16 : a, a1 = swap ? a : a + 16;
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
               : "r"(a0));
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
               : "r"(a1));
#else
  const int o0 = swap ? 4 : 0, o1 = swap ? 0 : 4;
  for (int c = 0; c < 4; ++c) {
    v[c] = p[o0 + c];
    v[4 + c] = p[o1 + c];
  }
#endif
}
// Whether record r (= n pk + m) of a staged uw block has its halves swapped.
BTAM_HD bool uw_swapped(int r) { return ((r >> 2) & 1) != 0; }
// FP64: the 16-byte quarter k of record r sits at quarter k ^ uw_xor64(r)
// of the record in a staged uw block.  A record is 64 bytes, so its
// quarters start on bank groups 16 (r & 1) + 4 k'; with the XOR over bits
// 1-2 of r the same quarter of records r mod 8 = 0..7 falls on eight
// different 4-bank groups, and the 128-bit shared loads of random records
// spread over all 32 banks.
BTAM_HD int uw_xor64(int r) { return (r >> 1) & 3; }
// 8 doubles of a 64-byte record in shared memory, quarters placed by x =
// uw_xor64(r) (four 128-bit shared loads; host: plain copy).
BTAM_HD void lds8(const double *p, int x, double (&v)[8]) {
#if defined(__CUDA_ARCH__)
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    asm volatile("ld.shared.v2.f64 {%0,%1}, [%2];"
                 : "=d"(v[2 * k]), "=d"(v[2 * k + 1])
                 : "r"(a + 16u * (unsigned)(k ^ x)));
#else
  for (int k = 0; k < 4; ++k) {
    v[2 * k] = p[2 * (k ^ x)];
    v[2 * k + 1] = p[2 * (k ^ x) + 1];
  }
#endif
}

template <class R> struct V3 {
  R x, y, z;
};
template <class R> BTAM_HD V3<R> mk3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R> BTAM_HD R dot3(const V3<R> &a, const V3<R> &b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class R> BTAM_HD R comp(const V3<R> &a, int k) {
  return k == 0 ? a.x : (k == 1 ? a.y : a.z);
}
template <class R> BTAM_HD V3<R> disp(const V3<R> &r, int k, R amount) {
  V3<R> o = r;
  if (k == 0) o.x += amount;
  else if (k == 1) o.y += amount;
  else o.z += amount;
  return o;
}

template <class R> BTAM_HD R my_sqrt(R v) { return std::sqrt(v); }
#if defined(__CUDA_ARCH__)
template <> __device__ __forceinline__ float my_sqrt<float>(float v) { return sqrtf(v); }
#endif

// A feature sum (a, L) with L symmetric stored (xx, yy, zz, xy, xz, yz).
template <class R> struct Feat {
  R a[3], l[6];
};

// A bilinear-form dual D of a feature sum X, stored as (Da, Lambda) with
// Lambda the full symmetric matrix such that B(X, Y) = Da.Ya + Lambda:Y_L:
//   Da = a/2, Lambda_kk = L_kk/2 - tr L/6, Lambda_kl = L_kl/2 (k != l).
template <class R> struct Dual {
  R a[3], d[3], o[3];  // d: xx,yy,zz; o: xy,xz,yz
};

template <class R, class S> BTAM_HD Dual<R> dual_of(const S *a, const S *l) {
  Dual<R> D;
  S tr = l[0] + l[1] + l[2];
  for (int k = 0; k < 3; ++k) D.a[k] = (R)(0.5 * a[k]);
  for (int k = 0; k < 3; ++k) D.d[k] = (R)(0.5 * l[k] - tr / 6.0);
  for (int k = 0; k < 3; ++k) D.o[k] = (R)(0.5 * l[3 + k]);
  return D;
}

// B(X, X) of a feature sum, evaluated in double.
template <class S> BTAM_HD double bself(const S *a, const S *l) {
  double aa = (double)a[0] * a[0] + (double)a[1] * a[1] + (double)a[2] * a[2];
  double ll = (double)l[0] * l[0] + (double)l[1] * l[1] + (double)l[2] * l[2] +
              2.0 * ((double)l[3] * l[3] + (double)l[4] * l[4] + (double)l[5] * l[5]);
  double tr = (double)l[0] + l[1] + l[2];
  return 0.5 * aa + 0.5 * ll - tr * tr / 6.0;
}

// B(X, Y) for two feature sums, in double.
template <class S> BTAM_HD double bpair(const S *a, const S *l, const S *b, const S *m) {
  double ab = (double)a[0] * b[0] + (double)a[1] * b[1] + (double)a[2] * b[2];
  double lm = (double)l[0] * m[0] + (double)l[1] * m[1] + (double)l[2] * m[2] +
              2.0 * ((double)l[3] * m[3] + (double)l[4] * m[4] + (double)l[5] * m[5]);
  double t1 = (double)l[0] + l[1] + l[2], t2 = (double)m[0] + m[1] + m[2];
  return 0.5 * ab + 0.5 * lm - t1 * t2 / 6.0;
}

// Lambda r
template <class R> BTAM_HD V3<R> lam_r(const Dual<R> &D, const V3<R> &r) {
  return mk3<R>(D.d[0] * r.x + D.o[0] * r.y + D.o[1] * r.z,
                D.o[0] * r.x + D.d[1] * r.y + D.o[2] * r.z,
                D.o[1] * r.x + D.o[2] * r.y + D.d[2] * r.z);
}

// Spline values at one displaced geometry.
template <class R> struct Geo {
  V3<R> r;
  R s, inv_s;     // |r|, 1/|r|
  R u, du, w, dw; // dipole and quadrupole splines and derivatives
};

// |r| and 1/|r| from |r|^2: IEEE sqrt and divide in double; in the FP32
// form one approximate reciprocal square root (a few ulp, far inside the
// form's 1e-6 relative energy budget).
BTAM_HD void norm_inv(double s2, double &s, double &inv) {
  s = std::sqrt(s2);
  inv = 1.0 / s;
}
BTAM_HD void norm_inv(float s2, float &s, float &inv) {
#if defined(__CUDA_ARCH__)
  inv = rsqrtf(s2);
#else
  inv = 1.0f / std::sqrt(s2);
#endif
  s = s2 * inv;
}

// The uw record of pair kind pk, segment m: a read-only global load, or a
// shared load when the view's uw block is staged in shared memory.
template <class R> BTAM_HD void ld_uw(const RadialView<R> &T, int pk, int m, R (&k)[8]) {
  ld8(uw_rec(T, pk, m), k);
}
BTAM_HD void ld_uw(const RadialViewS<float> &T, int pk, int m, float (&k)[8]) {
  lds8(uw_rec<float>(T, pk, m), uw_swapped(T.n * pk + m), k);
}
BTAM_HD void ld_uw(const RadialViewS<double> &T, int pk, int m, double (&k)[8]) {
  lds8(uw_rec<double>(T, pk, m), uw_xor64(T.n * pk + m), k);
}

// u, w of pair kind pk at one geometry (values and, when D, derivatives);
// returns the segment (m, p) for the pair-rule record of the same geometry.
template <class R, bool D, class TV = RadialView<R>>
BTAM_HD int geo_uw(Geo<R> &g, const V3<R> &r, const TV &T, int pk, R &p) {
  g.r = r;
  norm_inv(dot3(r, r), g.s, g.inv_s);
  const int m = seg_of<R>(T, g.s, p);
  R k[8];
  ld_uw(T, pk, m, k);
  if (D) {
    cub_vd(k, p, g.u, g.du);
    cub_vd(k + 4, p, g.w, g.dw);
  } else {
    g.u = cub_v(k, p);
    g.w = cub_v(k + 4, p);
    g.du = g.dw = (R)0;
  }
  return m;
}

// Pair-rule functions of pair kind pk at segment (m, p): phi, rho of the
// neighbour's species cj (rj) and, when WANT_I, of the centre's species ci
// (ri); derivatives when D.
template <class R, bool D, bool WANT_I>
BTAM_HD void pr_at(const RadialView<R> &T, int pk, int ci, int cj, int m, R p, R &ph, R &dph,
                   R &rj, R &drj, R &ri, R &dri) {
  const R *base = pr_rec(T, pk, m);
  R k[8];
  ld8(base, k);
  R r0 = (R)0, dr0 = (R)0, r1 = (R)0, dr1 = (R)0;
  if (D) {
    cub_vd(k, p, ph, dph);
    cub_vd(k + 4, p, r0, dr0);
  } else {
    ph = cub_v(k, p);
    r0 = cub_v(k + 4, p);
    dph = (R)0;
  }
  if (pk == 2 && (cj == 1 || (WANT_I && ci == 1))) {
    R h[4];
    ld4(base + 8, h);
    if (D) cub_vd(h, p, r1, dr1);
    else r1 = cub_v(h, p);
  }
  const bool jh = pk == 2 && cj == 1, ih = pk == 2 && ci == 1;
  rj = jh ? r1 : r0;
  drj = jh ? dr1 : dr0;
  ri = ih ? r1 : r0;
  dri = ih ? dr1 : dr0;
}

// A dual prepared for the six geometries r0 + a e_k that move along one
// axis: Lambda r, r^T Lambda r and Da.r at r0, so each displaced geometry
// costs a few FMAs instead of a full 3x3 contraction.
template <class R> struct DualAx {
  Dual<R> D;
  V3<R> Lr0;
  R rLr0, dar0;
};
template <class R> BTAM_HD DualAx<R> dual_ax(const Dual<R> &D, const V3<R> &r0) {
  DualAx<R> P;
  P.D = D;
  P.Lr0 = lam_r(D, r0);
  P.rLr0 = dot3(r0, P.Lr0);
  P.dar0 = D.a[0] * r0.x + D.a[1] * r0.y + D.a[2] * r0.z;
  return P;
}
// D . J(r) and D . f(r) at r = r0 + a e_k (g evaluated at that r).
template <class R>
BTAM_HD void dual_ax_at(const DualAx<R> &P, int k, R a, const Geo<R> &g, V3<R> &J, R &f) {
  const Dual<R> &D = P.D;
  V3<R> col = k == 0 ? mk3<R>(D.d[0], D.o[0], D.o[1])
                     : (k == 1 ? mk3<R>(D.o[0], D.d[1], D.o[2]) : mk3<R>(D.o[1], D.o[2], D.d[2]));
  R lkk = k == 0 ? D.d[0] : (k == 1 ? D.d[1] : D.d[2]);
  V3<R> Lr = mk3<R>(P.Lr0.x + a * col.x, P.Lr0.y + a * col.y, P.Lr0.z + a * col.z);
  R rLr = P.rLr0 + a * ((R)2 * comp(P.Lr0, k) + a * lkk);
  R dar = P.dar0 + a * D.a[k];
  R c = (g.du * dar + g.dw * rLr) * g.inv_s;
  R tw = (R)2 * g.w;
  J = mk3<R>(g.u * D.a[0] + c * g.r.x + tw * Lr.x, g.u * D.a[1] + c * g.r.y + tw * Lr.y,
             g.u * D.a[2] + c * g.r.z + tw * Lr.z);
  f = g.u * dar + g.w * rLr;
}

// D . f(r) alone at r = r0 + a e_k, formed as dual_ax_at forms it.
template <class R>
BTAM_HD R dual_ax_f(const DualAx<R> &P, int k, R a, const Geo<R> &g) {
  const Dual<R> &D = P.D;
  R lkk = k == 0 ? D.d[0] : (k == 1 ? D.d[1] : D.d[2]);
  R rLr = P.rLr0 + a * ((R)2 * comp(P.Lr0, k) + a * lkk);
  R dar = P.dar0 + a * D.a[k];
  return g.u * dar + g.w * rLr;
}

// D . f(r) with f(r) = (u r, w r r^T):  u (Da.r) + w (r^T Lambda r)
template <class R> BTAM_HD R dual_f(const Dual<R> &D, const Geo<R> &g) {
  V3<R> Da = mk3<R>(D.a[0], D.a[1], D.a[2]);
  V3<R> Lr = lam_r(D, g.r);
  return g.u * dot3(Da, g.r) + g.w * dot3(g.r, Lr);
}

// D . J(r) and D . f(r) together (one Lambda r).
template <class R> BTAM_HD void dual_Jf(const Dual<R> &D, const Geo<R> &g, V3<R> &J, R &f) {
  V3<R> Da = mk3<R>(D.a[0], D.a[1], D.a[2]);
  V3<R> Lr = lam_r(D, g.r);
  R dar = dot3(Da, g.r), rLr = dot3(g.r, Lr);
  R c = (g.du * dar + g.dw * rLr) * g.inv_s;
  R tw = (R)2 * g.w;
  J = mk3<R>(g.u * Da.x + c * g.r.x + tw * Lr.x, g.u * Da.y + c * g.r.y + tw * Lr.y,
             g.u * Da.z + c * g.r.z + tw * Lr.z);
  f = g.u * dar + g.w * rLr;
}

// D . J(r) with J = df/dr:  u Da + [(u'/s) Da.r + (w'/s) r^T Lambda r] r + 2 w Lambda r
template <class R> BTAM_HD V3<R> dual_J(const Dual<R> &D, const Geo<R> &g) {
  V3<R> Da = mk3<R>(D.a[0], D.a[1], D.a[2]);
  V3<R> Lr = lam_r(D, g.r);
  R c = (g.du * dot3(Da, g.r) + g.dw * dot3(g.r, Lr)) * g.inv_s;
  R tw = (R)2 * g.w;
  return mk3<R>(g.u * Da.x + c * g.r.x + tw * Lr.x,
                g.u * Da.y + c * g.r.y + tw * Lr.y,
                g.u * Da.z + c * g.r.z + tw * Lr.z);
}

// B(f, f) = u^2 s^2 / 2 + w^2 s^4 / 3 at one geometry, and its gradient
// [u u' s + u^2 + 2/3 w w' s^3 + 4/3 w^2 s^2] r.
template <class R> BTAM_HD R bff(const Geo<R> &g) {
  R s2 = g.s * g.s;
  return (R)0.5 * g.u * g.u * s2 + g.w * g.w * s2 * s2 / (R)3;
}
template <class R> BTAM_HD R bff_grad_coef(const Geo<R> &g) {
  R s2 = g.s * g.s;
  return g.u * g.du * g.s + g.u * g.u +
         ((R)2 / (R)3) * g.w * g.dw * s2 * g.s + ((R)4 / (R)3) * g.w * g.w * s2;
}

// Dual of X f(r0) (one feature scaled by X).
template <class R> BTAM_HD Dual<R> dual_feat(const Geo<R> &g, R X) {
  Dual<R> D;
  R hu = (R)0.5 * X * g.u, hw = (R)0.5 * X * g.w;
  R s2 = g.s * g.s;
  D.a[0] = hu * g.r.x; D.a[1] = hu * g.r.y; D.a[2] = hu * g.r.z;
  R t = X * g.w * s2 / (R)6;
  D.d[0] = hw * g.r.x * g.r.x - t;
  D.d[1] = hw * g.r.y * g.r.y - t;
  D.d[2] = hw * g.r.z * g.r.z - t;
  D.o[0] = hw * g.r.x * g.r.y;
  D.o[1] = hw * g.r.x * g.r.z;
  D.o[2] = hw * g.r.y * g.r.z;
  return D;
}

template <class R> BTAM_HD void feat_add(Feat<R> &F, const Geo<R> &g) {
  F.a[0] += g.u * g.r.x; F.a[1] += g.u * g.r.y; F.a[2] += g.u * g.r.z;
  F.l[0] += g.w * g.r.x * g.r.x; F.l[1] += g.w * g.r.y * g.r.y;
  F.l[2] += g.w * g.r.z * g.r.z; F.l[3] += g.w * g.r.x * g.r.y;
  F.l[4] += g.w * g.r.x * g.r.z; F.l[5] += g.w * g.r.y * g.r.z;
}

template <class R> BTAM_HD Dual<R> dual_sub(const Dual<R> &A, const Dual<R> &B) {
  Dual<R> D;
  for (int k = 0; k < 3; ++k) {
    D.a[k] = A.a[k] - B.a[k];
    D.d[k] = A.d[k] - B.d[k];
    D.o[k] = A.o[k] - B.o[k];
  }
  return D;
}
template <class R> BTAM_HD Dual<R> dual_flip(const Dual<R> &A) {
  Dual<R> D = A;
  D.a[0] = -A.a[0]; D.a[1] = -A.a[1]; D.a[2] = -A.a[2];
  return D;
}

// Per-site moment record written by pass 1 and read by pass 2 (kMomStride R,
// 32-byte aligned for vector loads):
//   [0] x_i F'(rho_i), [1] (H ? x_i : 1) F'(rho_i) (the occupancy-gradient
//   embedding factor of MgHx-mf-V-bulk.cpp:2299-2315), [2] beta_i, [3..7] 0;
//   then the bilinear-form duals of 8 feature sums, k = 0: G0, 1: H,
//   2 + d: G(d) for d = (axis, sign) in the order (x+, x-, y+, y-, z+, z-):
//   dual k's first eight components (a0 a1 a2 d0 d1 d2 o0 o1) at 8 + 8k and
//   its last one (o2) at 72 + k.
constexpr int kMomStride = 80;
constexpr int kDualG0 = 0, kDualH = 1, kDualGd = 2;

template <class R> BTAM_HD Dual<R> dual_from(const R (&h)[8], R o2) {
  Dual<R> D;
  D.a[0] = h[0]; D.a[1] = h[1]; D.a[2] = h[2];
  D.d[0] = h[3]; D.d[1] = h[4]; D.d[2] = h[5];
  D.o[0] = h[6]; D.o[1] = h[7]; D.o[2] = o2;
  return D;
}
template <class R, class S> BTAM_HD void store_dual(R *m, int k, const Dual<S> &D) {
  R *h = m + 8 + 8 * k;
  h[0] = (R)D.a[0]; h[1] = (R)D.a[1]; h[2] = (R)D.a[2];
  h[3] = (R)D.d[0]; h[4] = (R)D.d[1]; h[5] = (R)D.d[2];
  h[6] = (R)D.o[0]; h[7] = (R)D.o[1];
  m[72 + k] = (R)D.o[2];
}

// ---------------------------------------------------------------------------
// Pair kind for phi/u/w tables: Mg-Mg, H-H, else Mg-H (MgHx-ADP.cpp:881-888).
// Species codes: 0 = Mg, 1 = H.
BTAM_HD int pair_kind(int ci, int cj) { return ci == cj ? ci : 2; }

// ---------------------------------------------------------------------------
// B(X, Y) of two feature sums in the working type.
template <class R> BTAM_HD R bpair_r(const Feat<R> &x, const Feat<R> &y) {
  R ab = x.a[0] * y.a[0] + x.a[1] * y.a[1] + x.a[2] * y.a[2];
  R lm = x.l[0] * y.l[0] + x.l[1] * y.l[1] + x.l[2] * y.l[2] +
         (R)2 * (x.l[3] * y.l[3] + x.l[4] * y.l[4] + x.l[5] * y.l[5]);
  R t1 = x.l[0] + x.l[1] + x.l[2], t2 = y.l[0] + y.l[1] + y.l[2];
  return (R)0.5 * ab + (R)0.5 * lm - t1 * t2 / (R)6;
}

// The 12-point pair rule of an owned pair (u, j), once for both passes and
// both directions.  Pass 1 needs its raw sums; pass 2 needs the gradient
// pieces, which are linear in the embedding factors that pass 1 produces:
// with A = rho'_{s_j}/s, B = rho'_{s_u}/s, C = X phi'/(2 s) + X^2 dB(f,f)/ds
// / s at each point r (s = |r|), the radial coefficients of pass 2 are
//   c_self = w6 (x_u F'(rho_u) x_j A + C),   c_cros = w6 (x_j F'(rho_j) x_u B + C),
// so the record keeps sum A r, sum B r, sum C r and their sigma-direction
// sums over each side.  Layout (kPrRec R), stored as two arrays: the four
// pass-1 sums (kPr1 R per pair, compact so that pass 1's scattered reads
// stay in L2) and the pass-2 pieces (kPr2 R per pair, 32-byte aligned):
//   [0] sum rho_{s_u}, [1] sum rho_{s_j}, [2] sum phi, [3] sum B(f, f),
//   [4..6] sum A r, [7..9] sum B r, [10..12] sum C r,
//   [13..15] sum (A, B, C) sd over the u-moved points (sd = -+sqrt6 r_k),
//   [16..18] sum (A, B, C) sd over the j-moved points (sd = +-sqrt6 r_k),
//   [19] 0.
constexpr int kPr1 = 4, kPr2 = 16, kPrRec = kPr1 + kPr2;
template <class R, class TV>
BTAM_HD void pair_rule_record(const TV &T, const V3<R> &r0, R sig_u, R sig_j, R xu,
                              R xj, int cu, int cj, R (&rec)[kPrRec]) {
  const int pk = pair_kind(cu, cj);
  const R X = xu * xj;
#pragma unroll
  for (int c = 0; c < kPrRec; ++c) rec[c] = (R)0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const R amt = (side == 0 ? sig_u : -sig_j) * (R)kDelta6;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const R a = sg ? -amt : amt;
        Geo<R> g;
        R p;
        const int m = geo_uw<R, true>(g, disp(r0, k, a), T, pk, p);
        R rj, drj, ru, dru, ph, dph;
        pr_at<R, true, true>(T, pk, cu, cj, m, p, ph, dph, rj, drj, ru, dru);
        const R A = drj * g.inv_s, B = dru * g.inv_s;
        const R C = (R)0.5 * X * dph * g.inv_s + X * X * bff_grad_coef(g);
        rec[0] += ru;
        rec[1] += rj;
        rec[2] += ph;
        rec[3] += bff(g);
        rec[4] += A * g.r.x; rec[5] += A * g.r.y; rec[6] += A * g.r.z;
        rec[7] += B * g.r.x; rec[8] += B * g.r.y; rec[9] += B * g.r.z;
        rec[10] += C * g.r.x; rec[11] += C * g.r.y; rec[12] += C * g.r.z;
        // d r / d sigma along the moved site's axis: side 0 moves u, side 1 moves j
        const R sd = ((side == 0) == (sg != 0) ? -(R)kDelta6 : (R)kDelta6) * comp(g.r, k);
        const int o = side == 0 ? 13 : 16;
        rec[o] += A * sd;
        rec[o + 1] += B * sd;
        rec[o + 2] += C * sd;
      }
  }
}

// The four pass-1 sums of pair_rule_record alone ([0] sum rho_{s_u},
// [1] sum rho_{s_j}, [2] sum phi, [3] sum B(f, f)), from the same points
// and operations without their derivatives.  They depend on positions and
// widths only, so a run of evaluations at fixed positions and widths (the
// master equation's steps) can keep them.
template <class R, class TV>
BTAM_HD void pair_rule_sums(const TV &T, const V3<R> &r0, R sig_u, R sig_j, int cu, int cj,
                            R (&rec)[kPr1]) {
  const int pk = pair_kind(cu, cj);
#pragma unroll
  for (int c = 0; c < kPr1; ++c) rec[c] = (R)0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const R amt = (side == 0 ? sig_u : -sig_j) * (R)kDelta6;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const R a = sg ? -amt : amt;
        Geo<R> g;
        R p;
        const int m = geo_uw<R, false>(g, disp(r0, k, a), T, pk, p);
        R rj, drj, ru, dru, ph, dph;
        pr_at<R, false, true>(T, pk, cu, cj, m, p, ph, dph, rj, drj, ru, dru);
        rec[0] += ru;
        rec[1] += rj;
        rec[2] += ph;
        rec[3] += bff(g);
      }
  }
}

// The 12-point pair rule of pair (i, j): the rho, phi and B(f, f) sums over
// the points where the centre moves +-sqrt6 sigma_i e_k or the neighbour moves
// -+sqrt6 sigma_j e_k.  Returns x_j sum rho_{s_j} in *rho_j and, for the
// reverse pair (j, i) whose points are the same set negated, x_i sum rho_{s_i}
// in *rho_i when rho_i is not null.
template <class R, class TV>
BTAM_HD void pass1_pair_rule(const TV &T, const V3<R> &r0, R sig_i, R sig_j, R xi,
                             R xj, int ci, int cj, R &rho_j, R *rho_i, R &epair, R &ediag) {
  const int pk = pair_kind(ci, cj);
  const R X = xi * xj;
  R rho = 0, rhoi = 0, phi = 0, diag = 0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    R amt = (side == 0 ? sig_i : -sig_j) * (R)kDelta6;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        Geo<R> g;
        R p;
        const int m = geo_uw<R, false>(g, disp(r0, k, sg ? -amt : amt), T, pk, p);
        R ph, dph, rj, drj, ri, dri;
        if (rho_i) pr_at<R, false, true>(T, pk, ci, cj, m, p, ph, dph, rj, drj, ri, dri);
        else pr_at<R, false, false>(T, pk, ci, cj, m, p, ph, dph, rj, drj, ri, dri);
        rho += rj;
        if (rho_i) rhoi += ri;
        phi += ph;
        diag += bff(g);
      }
  }
  rho_j = xj * rho;
  if (rho_i) *rho_i = xi * rhoi;
  epair = (R)0.5 * X * phi;
  ediag = X * X * diag;
}

// ---------------------------------------------------------------------------
// Pass 1 per-pair moments in flat accumulator arrays (one lane per
// neighbour), in two parts so that few accumulators are live at once.
// Part I: the pair-rule sums, the centre point and the six
// neighbour-displaced points (-+3 sigma_j e_k); part II: the six
// centre-displaced points (+-3 sigma_i e_k).  Index layout of the flat
// pass-1 values (the order of SiteSums' fields up to the G(d) block):
constexpr int kP1Rho = 0, kP1Epair = 1, kP1Ediag = 2, kP1Cross = 3, kP1Sself = 4;
constexpr int kP1G0 = 5, kP1H = 14, kP1Gd = 23;  // 9 each; G(d) at kP1Gd + 9 d
constexpr int kP1Used = 77;
// Part I accumulates values [0, 23) except sself; part II values sself and
// [23, 77) at part-local index 0 (sself) and 1 + (v - 23).
constexpr int kP1PartI = 32, kP1PartII = 64;  // padded array lengths

// acc[base..base+8] += Xu r, Xw r r^T (feature scaled by X, as (a, L)).
template <class R> BTAM_HD void feat_acc(R *acc, int base, const Geo<R> &g, R X) {
  const R xu = X * g.u, xw = X * g.w;
  const R x = g.r.x, y = g.r.y, z = g.r.z;
  acc[base + 0] += xu * x;
  acc[base + 1] += xu * y;
  acc[base + 2] += xu * z;
  acc[base + 3] += xw * (x * x);
  acc[base + 4] += xw * (y * y);
  acc[base + 5] += xw * (z * z);
  acc[base + 6] += xw * (x * y);
  acc[base + 7] += xw * (x * z);
  acc[base + 8] += xw * (y * z);
}

// Part I without the pair rule: g0 += X f(r0), hsum += X sum_{6} f,
// cross += X^2 B(sum_6 f, f(r0)) over the neighbour-displaced points.
template <class R, class TV>
BTAM_HD void pass1_pair_part1(const TV &T, const V3<R> &r0, R sig_j, R X, int pk,
                              R *acc) {
  Geo<R> g0;
  R p;
  geo_uw<R, false>(g0, r0, T, pk, p);
  Feat<R> f0{};
  feat_add(f0, g0);
  Feat<R> hs{};
  const R amt_j = sig_j * (R)kDelta9;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int sg = 0; sg < 2; ++sg) {
      Geo<R> g;
      geo_uw<R, false>(g, disp(r0, k, sg ? amt_j : -amt_j), T, pk, p);
      feat_add(hs, g);
    }
  for (int c = 0; c < 3; ++c) {
    acc[kP1G0 + c] += X * f0.a[c];
    acc[kP1H + c] += X * hs.a[c];
  }
  for (int c = 0; c < 6; ++c) {
    acc[kP1G0 + 3 + c] += X * f0.l[c];
    acc[kP1H + 3 + c] += X * hs.l[c];
  }
  acc[kP1Cross] += X * X * bpair_r(hs, f0);
}

// Part II: G(d) += X f(r0 + d) for the six centre displacements d (part
// index 1 + 9 d + c) and sself += X^2 sum_d B(f, f) (part index 0).
template <class R, class TV>
BTAM_HD void pass1_pair_part2(const TV &T, const V3<R> &r0, R sig_i, R X, int pk,
                              R *acc) {
  const R amt_i = sig_i * (R)kDelta9;
  R ss = (R)0, p;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int sg = 0; sg < 2; ++sg) {
      Geo<R> g;
      geo_uw<R, false>(g, disp(r0, k, sg ? -amt_i : amt_i), T, pk, p);
      feat_acc(acc, 1 + 9 * (2 * k + sg), g, X);
      ss += bff(g);
    }
  acc[0] += X * X * ss;
}

// Part II for one axis k only (the FP64 form runs three of these, so that
// 19 accumulators are live instead of 55): G(d) for d = 2k, 2k + 1 at part
// index 1 + 9 (d - 2k) + c and the axis' share of sself at part index 0.
template <class R, class TV>
BTAM_HD void pass1_pair_part2_axis(const TV &T, const V3<R> &r0, R sig_i, R X, int pk, int k,
                                   R *acc) {
  const R amt_i = sig_i * (R)kDelta9;
  R ss = (R)0, p;
#pragma unroll
  for (int sg = 0; sg < 2; ++sg) {
    Geo<R> g;
    geo_uw<R, false>(g, disp(r0, k, sg ? -amt_i : amt_i), T, pk, p);
    feat_acc(acc, 1 + 9 * sg, g, X);
    ss += bff(g);
  }
  acc[0] += X * X * ss;
}

// Flat pass-1 value of part II's local index t.
BTAM_HD int p1_part2_value(int t) { return t == 0 ? kP1Sself : kP1Gd + (t - 1); }

// Position of flat pass-1 value v in SiteSums viewed as an array of doubles.
BTAM_HD int p1_site_slot(int v) {
  if (v < kP1Gd) return v;
  const int d = (v - kP1Gd) / 9, c = (v - kP1Gd) % 9;
  return c < 3 ? kP1Gd + 3 * d + c : kP1Gd + 18 + 6 * d + (c - 3);
}

// ---------------------------------------------------------------------------
// Pass 2: contributions of neighbour j to the residuals of site u.
// r0 = q_u - q_j.  mu, mj: moment records of u and of j's owner.
// embq_u = x_u F'(rho_u); embq_j, embx_j likewise for j; omega = beta_j/beta_u.
// Outputs (added):  gq (3): dS/dq_u / beta_u pieces, gs: d/dsigma_u,
// gx: d/dx_u of V0_j (cross term only; the self occupancy term is per site).
template <class R> struct Pass2Out {
  R gq[3];
  R gs;
  R gx;
};

// Moment-record readers: plain loads (host, shared memory) or read-only
// cached global loads (device, neighbour records).
template <class R> BTAM_HD R ld_plain(const R *p) { return *p; }
template <class R> BTAM_HD R ld_ro(const R *p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}
// A moment record in global memory (RO: read-only cached vector loads) or in
// host / shared memory (plain loads).  The o2 components of its eight duals
// are read once, with the record.
template <class R, bool RO> struct MomRec {
  const R *m;
  R tail[8];
  BTAM_HD explicit MomRec(const R *m_) : m(m_) {
    if (RO) ld8(m + 72, tail);
    else cp8(m + 72, tail);
  }
  BTAM_HD R scalar(int c) const { return RO ? ld_ro(m + c) : ld_plain(m + c); }
  BTAM_HD Dual<R> dual(int k) const {
    R h[8];
    if (RO) ld8(m + 8 + 8 * k, h);
    else cp8(m + 8 + 8 * k, h);
    return dual_from(h, tail[k]);
  }
};

// The two parts of pair (u, j), unweighted: self = the terms of
// dV0_u/d(q_u, sigma_u) that pair j carries, cros = dV0_j/d(q_u, sigma_u,
// x_u), the reference's evaluate_DV0_i_Dq_u(u, j) and
// evaluate_DV0_i_Dxi_u(u, j) (MgHx-mf-V-bulk.cpp:1823-2098, 2102-2325).
template <class R> struct Pass2Parts {
  R self_q[3], self_s;
  R cros_q[3], cros_s, cros_x;
};

template <class R, class MU, class MJ>
BTAM_HD void pass2_pair_parts(const RadialView<R> &T, const V3<R> &r0, R sig_u,
                              R sig_j, R xu, R xj, int cu, int cj, R embq_u,
                              R embq_j, R embx_j, const MU &mu, const MJ &mj,
                              Pass2Parts<R> &P) {
  const int pk = pair_kind(cu, cj);
  const R X = xu * xj;
  const R w6 = (R)kW6, w9 = (R)kW9;

  R self_q[3] = {0, 0, 0}, self_s = 0;
  R cros_q[3] = {0, 0, 0}, cros_s = 0, cros_x = 0;

  // ---- 12-point pair rule geometries: u-displaced (C) and j-displaced (D)
  {
    R rho_sum = 0, phi_sum = 0, bff_sum = 0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      R amt = (side == 0 ? sig_u : -sig_j) * (R)kDelta6;
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int sg = 0; sg < 2; ++sg) {
          R a = sg ? -amt : amt;
          Geo<R> g;
          R p;
          const int m = geo_uw<R, true>(g, disp(r0, k, a), T, pk, p);
          R rj, drj, ru, dru, ph, dph;
          pr_at<R, true, true>(T, pk, cu, cj, m, p, ph, dph, rj, drj, ru, dru);
          R bc = bff_grad_coef(g);
          // radial coefficient of d/dr for each piece
          R c_self = w6 * (embq_u * xj * drj * g.inv_s + (R)0.5 * X * dph * g.inv_s + X * X * bc);
          R c_cros = w6 * (embq_j * xu * dru * g.inv_s + (R)0.5 * X * dph * g.inv_s + X * X * bc);
          self_q[0] += c_self * g.r.x; self_q[1] += c_self * g.r.y; self_q[2] += c_self * g.r.z;
          cros_q[0] += c_cros * g.r.x; cros_q[1] += c_cros * g.r.y; cros_q[2] += c_cros * g.r.z;
          if (side == 0) {  // only u-displaced points depend on sigma_u
            R sd = (sg ? -(R)kDelta6 : (R)kDelta6) * comp(g.r, k);
            self_s += c_self * sd;
            cros_s += c_cros * sd;
          }
          rho_sum += ru;
          phi_sum += ph;
          bff_sum += bff(g);
        }
    }
    cros_x += w6 * (embx_j * rho_sum + (R)0.5 * xj * phi_sum + (R)2 * X * xj * bff_sum);
  }

  // ---- triplet geometries
  Geo<R> gc;
  {
    R p;
    geo_uw<R, true>(gc, r0, T, pk, p);
  }
  const Dual<R> Xf0 = dual_feat(gc, X);  // dual of X f(r0)

  const R sfac = (R)2 * w9 * X;
  // A: u displaced by +-3 sigma_u e_k.  Self centre-displaced term (S4); the
  // neighbour-displaced term of j's energy (C5) and its occupancy gradient
  // (X5) use fixed duals, so they go through the axis-displacement form.
  Feat<R> FA{};
  {
    const Dual<R> Dj_g0 = mj.dual(kDualG0);
    const Dual<R> Dc5 = dual_sub(dual_flip(Dj_g0), Xf0);
    const DualAx<R> c5 = dual_ax(Dc5, r0);
    const DualAx<R> x5 = dual_ax(dual_sub(Dc5, Xf0), r0);
    const R amt = sig_u * (R)kDelta9;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const R a = sg ? -amt : amt;
        Geo<R> g;
        R p;
        geo_uw<R, true>(g, disp(r0, k, a), T, pk, p);
        feat_add(FA, g);
        R hb = (R)0.5 * X * bff_grad_coef(g);
        V3<R> v4 = dual_J(mu.dual(kDualGd + 2 * k + sg), g);  // S4
        V3<R> v5, vx;
        R f5, fx;
        dual_ax_at(c5, k, a, g, v5, f5);  // C5
        dual_ax_at(x5, k, a, g, vx, fx);  // X5: (P Dj.g0 - 2X dual(f0)) . f(r_A)
        V3<R> s4 = mk3<R>(v4.x - hb * g.r.x, v4.y - hb * g.r.y, v4.z - hb * g.r.z);
        self_q[0] += sfac * s4.x; self_q[1] += sfac * s4.y; self_q[2] += sfac * s4.z;
        cros_q[0] += sfac * v5.x; cros_q[1] += sfac * v5.y; cros_q[2] += sfac * v5.z;
        R sd = sg ? -(R)kDelta9 : (R)kDelta9;
        self_s += sfac * comp(s4, k) * sd;
        cros_s += sfac * comp(v5, k) * sd;
        cros_x += (R)2 * w9 * xj * fx;
      }
  }
  // B: j displaced by -+3 sigma_j e_k (centre j displaced by +-3 sigma_j e_k
  // in j's frame).  Self neighbour-displaced term (S5, fixed dual) and j's
  // centre-displaced term (C4) with its occupancy gradient (X4).
  Feat<R> FB{};
  {
    const DualAx<R> s5 = dual_ax(dual_sub(mu.dual(kDualG0), Xf0), r0);
    const R amt = sig_j * (R)kDelta9;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const R a = sg ? amt : -amt;
        Geo<R> g;
        R p;
        geo_uw<R, true>(g, disp(r0, k, a), T, pk, p);
        feat_add(FB, g);
        V3<R> v5;
        R f5;
        dual_ax_at(s5, k, a, g, v5, f5);
        self_q[0] += sfac * v5.x; self_q[1] += sfac * v5.y; self_q[2] += sfac * v5.z;
        const Dual<R> Pj = dual_flip(mj.dual(kDualGd + 2 * k + sg));
        V3<R> v4;
        R f4;
        dual_Jf(Pj, g, v4, f4);
        R hb = (R)0.5 * X * bff_grad_coef(g);
        cros_q[0] += sfac * (v4.x - hb * g.r.x);
        cros_q[1] += sfac * (v4.y - hb * g.r.y);
        cros_q[2] += sfac * (v4.z - hb * g.r.z);
        cros_x += (R)2 * w9 * xj * (f4 - X * bff(g));
      }
  }
  // centre-geometry pieces of S5 and C5:  (D_H - X dual(F)) . J(r0)
  {
    Dual<R> dFB = dual_of<R, R>(FB.a, FB.l);
    Dual<R> dFA = dual_of<R, R>(FA.a, FA.l);
    for (int k = 0; k < 3; ++k) {
      dFB.a[k] *= X; dFB.d[k] *= X; dFB.o[k] *= X;
      dFA.a[k] *= X; dFA.d[k] *= X; dFA.o[k] *= X;
    }
    const Dual<R> Dj_h = mj.dual(kDualH);
    V3<R> vs = dual_J(dual_sub(mu.dual(kDualH), dFB), gc);
    V3<R> vc = dual_J(dual_sub(dual_flip(Dj_h), dFA), gc);
    self_q[0] += sfac * vs.x; self_q[1] += sfac * vs.y; self_q[2] += sfac * vs.z;
    cros_q[0] += sfac * vc.x; cros_q[1] += sfac * vc.y; cros_q[2] += sfac * vc.z;
    // X5 second piece: (P Dj.h) . f0  (its -2X B(F_A, f0) part was summed in
    // the A loop above)
    cros_x += (R)2 * w9 * xj * dual_f(dual_flip(Dj_h), gc);
  }

  for (int k = 0; k < 3; ++k) {
    P.self_q[k] = self_q[k];
    P.cros_q[k] = cros_q[k];
  }
  P.self_s = self_s;
  P.cros_s = cros_s;
  P.cros_x = cros_x;
}

// Both parts of pair (u, j) weighted into u's residual: self + omega cros,
// omega = beta_j / beta_u.
template <class R, class MU, class MJ>
BTAM_HD void pass2_pair(const RadialView<R> &T, const V3<R> &r0, R sig_u,
                        R sig_j, R xu, R xj, int cu, int cj, R embq_u,
                        R embq_j, R embx_j, R omega, const MU &mu,
                        const MJ &mj, Pass2Out<R> &o) {
  Pass2Parts<R> P;
  pass2_pair_parts(T, r0, sig_u, sig_j, xu, xj, cu, cj, embq_u, embq_j, embx_j, mu, mj, P);
  for (int k = 0; k < 3; ++k) o.gq[k] += P.self_q[k] + omega * P.cros_q[k];
  o.gs += P.self_s + omega * P.cros_s;
  o.gx += omega * P.cros_x;
}

// ---------------------------------------------------------------------------
// Pass 2, one undirected pair {u, j}: the contributions of j to u's residuals
// (ou, exactly what pass2_pair returns for (u, j)) and of u to j's residuals
// (oj, what pass2_pair returns for (j, u)), from the 25 geometries of (u, j)
// only.  The two directions share every geometry: those of (j, u) are the
// negated ones of (u, j) with the pair-rule sides and the triplet loops
// swapped (j's centre-displaced points are u's neighbour-displaced points).
// Position gradients follow from translation invariance of each pair term,
//   dV0_j/dq_j|u = -dV0_j/dq_u|u,   dV0_u/dq_j|j = -dV0_u/dq_u|j,
// so oj.gq = -cros_q - omega_ju self_q; the width and occupancy gradients of
// j take the sigma_j and x_u derivatives of the same terms (rself_s, rcros_s,
// rcros_x).  mu, mj: moment records of u and of j's owner; omega_uj =
// beta_j / beta_u, omega_ju = beta_u / beta_j; pr: the pair's record from
// pair_rule_record (its 12 pair-rule points were evaluated once, in pass 1;
// only the 13 triplet geometries are evaluated here).
// XO: the occupancy gradients only (ou.gx, oj.gx), the chemical potentials
// of the master equation: the same x terms from the same operations, the
// values at the 13 geometries without their derivatives, no position or
// width terms (ou.gq, ou.gs, oj.gq, oj.gs are left as they are).
template <class R, class MU, class MJ, class TV, bool XO = false>
BTAM_HD void pass2_pair_sym(const TV &T, const V3<R> &r0, R sig_u, R sig_j, R xu,
                            R xj, int cu, int cj, R embq_u, R embx_u, R embq_j, R embx_j,
                            R omega_uj, R omega_ju, const MU &mu, const MJ &mj,
                            const R (&pr)[kPrRec], Pass2Out<R> &ou, Pass2Out<R> &oj) {
  const int pk = pair_kind(cu, cj);
  const R X = xu * xj;
  const R w6 = (R)kW6, w9 = (R)kW9;

  // u's view: d/dq_u and d/dsigma_u of V0_u (self) and V0_j (cros), d/dx_u of V0_j
  R self_q[3] = {0, 0, 0}, self_s = 0;
  R cros_q[3] = {0, 0, 0}, cros_s = 0, cros_x = 0;
  // j's view: d/dsigma_j of V0_j (rself_s) and of V0_u (rcros_s), d/dx_j of V0_u
  R rself_s = 0, rcros_s = 0, rcros_x = 0;

  // ---- 12-point pair rule, from the pair's record (pair_rule_record)
  {
    if constexpr (!XO) {
      const R ku = embq_u * xj, kj = embq_j * xu;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        self_q[c] = w6 * (ku * pr[4 + c] + pr[10 + c]);
        cros_q[c] = w6 * (kj * pr[7 + c] + pr[10 + c]);
      }
      self_s = w6 * (ku * pr[13] + pr[15]);
      cros_s = w6 * (kj * pr[14] + pr[15]);
      rself_s = w6 * (kj * pr[17] + pr[18]);
      rcros_s = w6 * (ku * pr[16] + pr[18]);
    }
    cros_x = w6 * (embx_j * pr[0] + (R)0.5 * xj * pr[2] + (R)2 * X * xj * pr[3]);
    rcros_x = w6 * (embx_u * pr[1] + (R)0.5 * xu * pr[2] + (R)2 * X * xu * pr[3]);
  }

  // ---- triplet geometries
  Geo<R> gc;
  {
    R p;
    geo_uw<R, !XO>(gc, r0, T, pk, p);
  }
  const Dual<R> Xf0 = dual_feat(gc, X);
  const R sfac = (R)2 * w9 * X;
  // A: u displaced by +-3 sigma_u e_k (j's neighbour-displaced points)
  Feat<R> FA{};
  {
    const Dual<R> Dj_g0 = mj.dual(kDualG0);
    const Dual<R> Dc5 = dual_sub(dual_flip(Dj_g0), Xf0);
    const DualAx<R> c5 = dual_ax(Dc5, r0);
    const DualAx<R> x5 = dual_ax(dual_sub(Dc5, Xf0), r0);
    const R amt = sig_u * (R)kDelta9;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const R a = sg ? -amt : amt;
        Geo<R> g;
        R p;
        geo_uw<R, !XO>(g, disp(r0, k, a), T, pk, p);
        if constexpr (XO) {
          const R fx = dual_ax_f(x5, k, a, g);
          const R f4u = dual_f(mu.dual(kDualGd + 2 * k + sg), g);
          cros_x += (R)2 * w9 * xj * fx;
          rcros_x += (R)2 * w9 * xu * (f4u - X * bff(g));
        } else {
          feat_add(FA, g);
          R hb = (R)0.5 * X * bff_grad_coef(g);
          V3<R> v4;
          R f4u;
          dual_Jf(mu.dual(kDualGd + 2 * k + sg), g, v4, f4u);  // S4
          V3<R> v5, vx;
          R f5, fx;
          dual_ax_at(c5, k, a, g, v5, f5);  // C5
          dual_ax_at(x5, k, a, g, vx, fx);  // X5
          V3<R> s4 = mk3<R>(v4.x - hb * g.r.x, v4.y - hb * g.r.y, v4.z - hb * g.r.z);
          self_q[0] += sfac * s4.x; self_q[1] += sfac * s4.y; self_q[2] += sfac * s4.z;
          cros_q[0] += sfac * v5.x; cros_q[1] += sfac * v5.y; cros_q[2] += sfac * v5.z;
          R sd = sg ? -(R)kDelta9 : (R)kDelta9;
          self_s += sfac * comp(s4, k) * sd;
          cros_s += sfac * comp(v5, k) * sd;
          cros_x += (R)2 * w9 * xj * fx;
          // j's view: u's centre-displaced term as a function of x_j
          rcros_x += (R)2 * w9 * xu * (f4u - X * bff(g));
        }
      }
  }
  // B: j displaced by -+3 sigma_j e_k (j's centre-displaced points)
  Feat<R> FB{};
  {
    const Dual<R> Du_g0 = mu.dual(kDualG0);
    const DualAx<R> s5 = dual_ax(dual_sub(Du_g0, Xf0), r0);
    const DualAx<R> xf = dual_ax(Xf0, r0);
    const R amt = sig_j * (R)kDelta9;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const R a = sg ? amt : -amt;
        Geo<R> g;
        R p;
        geo_uw<R, !XO>(g, disp(r0, k, a), T, pk, p);
        if constexpr (XO) {
          const R f5 = dual_ax_f(s5, k, a, g);
          const R fxf = dual_ax_f(xf, k, a, g);
          const R f4 = dual_f(dual_flip(mj.dual(kDualGd + 2 * k + sg)), g);
          R bffg = bff(g);
          cros_x += (R)2 * w9 * xj * (f4 - X * bffg);
          rcros_x += (R)2 * w9 * xu * (f5 - fxf);
        } else {
          feat_add(FB, g);
          V3<R> v5, vxf;
          R f5, fxf;
          dual_ax_at(s5, k, a, g, v5, f5);  // S5
          dual_ax_at(xf, k, a, g, vxf, fxf);
          self_q[0] += sfac * v5.x; self_q[1] += sfac * v5.y; self_q[2] += sfac * v5.z;
          const Dual<R> Pj = dual_flip(mj.dual(kDualGd + 2 * k + sg));
          V3<R> v4;
          R f4;
          dual_Jf(Pj, g, v4, f4);  // C4
          R hb = (R)0.5 * X * bff_grad_coef(g);
          V3<R> c4 = mk3<R>(v4.x - hb * g.r.x, v4.y - hb * g.r.y, v4.z - hb * g.r.z);
          cros_q[0] += sfac * c4.x; cros_q[1] += sfac * c4.y; cros_q[2] += sfac * c4.z;
          R bffg = bff(g);
          cros_x += (R)2 * w9 * xj * (f4 - X * bffg);
          R sd = sg ? (R)kDelta9 : -(R)kDelta9;
          rself_s += sfac * comp(c4, k) * sd;
          rcros_s += sfac * comp(v5, k) * sd;
          // j's view: u's neighbour-displaced term as a function of x_j
          rcros_x += (R)2 * w9 * xu * (f5 - fxf);
        }
      }
  }
  // centre-geometry pieces
  {
    const Dual<R> Dj_h = mj.dual(kDualH);
    const Dual<R> Du_h = mu.dual(kDualH);
    if constexpr (!XO) {
      Dual<R> dFB = dual_of<R, R>(FB.a, FB.l);
      Dual<R> dFA = dual_of<R, R>(FA.a, FA.l);
      for (int k = 0; k < 3; ++k) {
        dFB.a[k] *= X; dFB.d[k] *= X; dFB.o[k] *= X;
        dFA.a[k] *= X; dFA.d[k] *= X; dFA.o[k] *= X;
      }
      V3<R> vs = dual_J(dual_sub(Du_h, dFB), gc);
      V3<R> vc = dual_J(dual_sub(dual_flip(Dj_h), dFA), gc);
      self_q[0] += sfac * vs.x; self_q[1] += sfac * vs.y; self_q[2] += sfac * vs.z;
      cros_q[0] += sfac * vc.x; cros_q[1] += sfac * vc.y; cros_q[2] += sfac * vc.z;
    }
    cros_x += (R)2 * w9 * xj * dual_f(dual_flip(Dj_h), gc);
    rcros_x += (R)2 * w9 * xu * dual_f(Du_h, gc);
  }

  if constexpr (!XO) {
    for (int k = 0; k < 3; ++k) {
      ou.gq[k] += self_q[k] + omega_uj * cros_q[k];
      oj.gq[k] += -cros_q[k] - omega_ju * self_q[k];
    }
    ou.gs += self_s + omega_uj * cros_s;
    oj.gs += rself_s + omega_ju * rcros_s;
  }
  ou.gx += omega_uj * cros_x;
  oj.gx += omega_ju * rcros_x;
}

// ---------------------------------------------------------------------------
// Per-site epilogue of pass 1, in double.  Inputs are the raw sums over the
// site's active neighbours (the pass-1 values, kP1Rho ... kP1Gd).
struct SiteSums {
  double rho, epair, ediag, cross, sself;
  double g0a[3], g0l[6], ha[3], hl[6];
  double gda[6][3], gdl[6][6];
};

struct SiteResult {
  double rho, V0, S0, selfx;
};

// Physical constants of the reference (Macros.hpp:846-854).
constexpr double kHbar = 6.5821192815E-4;   // eV ps
constexpr double kUma = 103.4993333E-6;     // eV A^-2 ps^2 per amu

// Energy of one site:  V0_i = x_i F(rho) + E_pair + E_angular
// (evaluate_V0_i_adp_MgHx, MgHx-mf-V-bulk.cpp:791-953), its free entropy
// S0_i (evaluate_S0_i_adp_MgHx, 957-1142), dV0_i/dx_i, and the moment
// record for pass 2 (layout at kMomStride).  In two parts so that a warp can
// run them on several lanes: site_dual forms dual k of the record (k = 0:
// G0, 1: H, 2 + d: G(d)) and returns B(G(d), G(d)) for the G(d) duals;
// site_scalars takes bgd = sum_d B(G(d), G(d)) (summed in d order) and does
// the rest.
template <class M> BTAM_HD double site_dual(const SiteSums &S, int k, M *mom) {
  const double *a = k == 0 ? S.g0a : (k == 1 ? S.ha : S.gda[k - 2]);
  const double *l = k == 0 ? S.g0l : (k == 1 ? S.hl : S.gdl[k - 2]);
  if (mom) store_dual(mom, k, dual_of<double, double>(a, l));
  return k >= 2 ? bself(a, l) : 0.0;
}

template <class M>
BTAM_HD void site_scalars(const SiteSums &S, double bgd, const SplineView<double> &emb,
                          double xi, int code, double beta, double gamma, double sigma,
                          double mass, SiteResult &res, M *mom) {
  const double rho = kW6 * S.rho;
  double F, dF;
  spline_vd(emb, rho, F, dF);
  const double e_pair = kW6 * S.epair;
  const double e_diag = kW6 * S.ediag;
  const double e_id = kW9 * (bgd - S.sself);
  const double e_jd = 2.0 * kW9 * (bpair(S.ha, S.hl, S.g0a, S.g0l) - S.cross);
  const double e_ang = e_id + e_jd + e_diag;
  const double V0 = xi * F + e_pair + e_ang;
  res.rho = rho;
  res.V0 = V0;
  // dV0_i/dx_i: H embedding F(rho) (2299-2302); Mg has none (2312-2315);
  // pair and angular terms are linear / quadratic in x_i.
  res.selfx = (code == 1 ? F : 0.0) + (e_pair + 2.0 * e_ang) / xi;
  // S0_i = -log Z0 + beta (1/(2 beta) + V0) - gamma x~
  double m = kUma * xi * mass;
  double logZ = 3.0 * std::log((sigma * std::sqrt(m / beta)) / kHbar);
  if (xi < 1.0) logZ += std::log(1.0 / (1.0 - xi));
  double gx = (code == 1) ? gamma * (xi > 0.9999 ? 0.9999 : xi) : 0.0;
  res.S0 = -logZ + beta * (1.0 / (2.0 * beta) + V0) - gx;
  if (mom) {
    mom[0] = (M)(xi * dF);
    mom[1] = (M)((code == 1 ? xi : 1.0) * dF);
    mom[2] = (M)beta;
    for (int c = 3; c < 8; ++c) mom[c] = (M)0;
  }
}

template <class M>
BTAM_HD void site_epilogue(const SiteSums &S, const SplineView<double> &emb,
                           double xi, int code, double beta, double gamma,
                           double sigma, double mass, SiteResult &res, M *mom) {
  double bgd = 0.0;
  for (int k = 0; k < 8; ++k) {
    const double b = site_dual(S, k, mom);
    if (k >= 2) bgd += b;
  }
  site_scalars(S, bgd, emb, xi, code, beta, gamma, sigma, mass, res, mom);
}

// Residual epilogue of pass 2 for site u (H sites also get the occupancy
// entropy terms; non-H sites carry no occupancy residual):
//   R_sigma -= 3 / (beta sigma),   R_x = selfx + sum - (3/(2x) + [x<1]/(1-x))/beta
//                                        - [x<0.9999] gamma/beta
BTAM_HD void residual_epilogue(double sigma, double x, int code, double beta,
                               double gamma, double selfx, double &rs,
                               double &rx) {
  rs -= 3.0 / (beta * sigma);
  if (code == 1) {
    double dlogz = 3.0 / (2.0 * x) + (x < 1.0 ? 1.0 / (1.0 - x) : 0.0);
    rx += selfx - dlogz / beta;
    if (x < 0.9999) rx -= gamma / beta;
  } else {
    rx = 0.0;
  }
}

}  // namespace btam
