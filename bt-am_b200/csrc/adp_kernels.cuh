// Launchers of the two-pass mean-field ADP kernels.
#pragma once

#include <cuda_runtime.h>

#include "adp_core.cuh"

namespace btam {

// Packed copy of what the FP32C kernels read about a neighbour, one 32-byte
// sector per site (made by launch_pass1 from pos / xb / code): the position
// in double, sigma with the species in its sign (negative: H), and the
// occupancy as the kernels use it, or -1 when the site is empty (occupancy
// below min_occupancy, decided in double).
struct __align__(32) Site32 {
  double x, y, z;
  float sig_code, occ;
};
// beta and owner of a site, for the pass-2 pair kernel.
struct __align__(16) SiteB {
  double beta;
  int owner, pad;
};
// Packed copy of what the FP64 kernels read about a neighbour, one 64-byte
// row (two sectors) per site (made by launch_pass1 from pos / xb / code /
// owner): position and sigma, then occupancy, species, owner and beta.
struct __align__(64) Site64 {
  double x, y, z, sigma;
  double occ;
  int code, owner;
  double beta, pad;
};

// Device view of one system for an evaluation.  Site arrays cover real sites
// then periodic images ("all sites"); per-site outputs cover real sites.
template <class R> struct EvalArgs {
  int n_real;
  int n_all = 0;        // real sites + images (rows of the site arrays)
  Site32 *s32 = nullptr;  // FP32C: packed neighbour data [all] (nullptr: unpacked)
  SiteB *sb = nullptr;    // FP32C: beta and owner [all]
  Site64 *s64 = nullptr;  // FP64: packed neighbour rows [all] (nullptr: unpacked)
  const double4 *pos;   // x, y, z, sigma            [all]
  const double2 *xb;    // occupancy x, beta         [all]
  const int *code;      // 0 = Mg, 1 = H             [all]
  const int *owner;     // real site of each row     [all]
  const double *gamma;  // chemical multiplier       [real]
  const int *offs;      // CSR offsets               [real + 1]
  const int *idx;       // neighbour indices (all-sites numbering)
  RadialView<R> T;      // radial tables in R (per-segment records)
  SplineView<double> emb[2];  // embedding F (FP64) for Mg, H
  double mass[2];             // Mg, H element masses
  R *mom;                     // kMomStride per real site
  double *rho, *V0, *S0, *selfx;  // [real]
  double *Rq, *Rs, *Rx;           // [3*real], [real], [real]
  int *err;
  // Occupancy gradients only (the master equation's chemical potentials):
  // with the undirected variants, pass 2 forms R_x alone and writes R_q and
  // R_sigma as 0, and the pair-rule kernel forms only the four pass-1 sums
  // of each pair (every pair, occupied or not: they do not depend on the
  // occupancies).  recs_ready: those sums are already in prec1 from an
  // earlier launch at the same positions and widths, so pass 1 skips the
  // pair-rule kernel.  Both are ignored by the directed variants.
  int x_only = 0;
  int recs_ready = 0;
  // Sites to evaluate (1 per real site; nullptr: all): a served round of a
  // batch evaluates only the systems that asked.  Every pair and triplet of
  // a system lies within it, so a site that is off is skipped whole.
  const unsigned char *site_on = nullptr;
  // undirected pass 2 (optional; nullptr / 0 when absent)
  const int *rev = nullptr;    // reverse slot of each real-site slot, -1 if none
  const int *own_p = nullptr;  // owned slots
  const int *own_u = nullptr;  // their sites
  int n_own = 0;
  R *pbuf = nullptr;           // 4 R per slot: gq[3], gs (pass-2 contributions)
  R *pgx = nullptr;            // 1 R per slot: gx
  // pair-rule records of the owned pairs (pair_rule_record: kPr1 R each in
  // prec1, the other kPr2 in prec2) and each slot's owned pair and direction
  // (2 t + 0 owned slot, + 1 its reverse)
  R *prec1 = nullptr, *prec2 = nullptr;
  const int *slot_own = nullptr;
};

// Pass 1: rho-bar, V0, S0, dV0/dx (self) and the moment record of every
// real site.  Pass 2: residuals of every real site.  `variant` picks the
// block shape / register cap (0 = default; see kPass1Variants below); pass 1
// also takes the pass-2 variant, because an undirected pass 2 needs the
// pair-rule records that pass 1 then makes.
// `mid`, when given, is recorded between a pass's pair kernel and its site
// kernel (at the start when the pass has no pair kernel), for per-kernel
// timing.
template <class R>
cudaError_t launch_pass1(const EvalArgs<R> &a, cudaStream_t st, int variant = 0,
                         int pass2_variant = 0, cudaEvent_t mid = nullptr);
template <class R>
cudaError_t launch_pass2(const EvalArgs<R> &a, cudaStream_t st, int variant = 0,
                         cudaEvent_t mid = nullptr);
// variant = shape | kPersistent (persistent grid of resident blocks)
//           [| kUndirected: pass 1 takes its pair-rule sums, pass 2 its
//            whole per-pair work, from one evaluation per undirected pair]
// pass-1 shapes (warps per block, min blocks per SM, lanes per site):
// (4,-,32), (4,5,8), (4,4,16), (8,2,16), (4,5,16), (4,3,16)
constexpr int kPass1Variants = 6;
constexpr int kPass2Variants = 6;  // shapes (4,-), (4,3), (4,4), (4,5), (8,2), (2,8)
// undirected pair kernel (threads, min blocks): (128,-), (128,5), (128,4),
// (256,2), then one block of 512 or 384 threads per SM with the uw tables in
// shared memory (always persistent), then (128,3)
constexpr int kPass2UVariants = 7;
constexpr int kPersistent = 8;
constexpr int kUndirected = 16;
inline bool valid_variants(int v1, int v2) {
  if (v1 < 0 || v2 < 0 || (v1 & ~(2 * kUndirected - 1)) != 0 ||
      (v2 & ~(2 * kUndirected - 1)) != 0)
    return false;
  const int s2 = v2 & (kPersistent - 1);
  return (v1 & (kPersistent - 1)) < kPass1Variants &&
         s2 < ((v2 & kUndirected) ? kPass2UVariants : kPass2Variants);
}

// Undirected pass 2 in two launches: the pair kernel (one thread per owned
// slot: both directions of the pair into the slot buffer) and the site
// kernel (one warp per site: the sum over its slots and the epilogue).
// Needs a.rev, a.own_p, a.own_u, a.pbuf, a.prec1/2 and a.slot_own; the launchers
// fall back to the directed default when they are absent.
// Layout (in R) of the undirected kernels' buffer: the slot 4-vectors (4 per
// slot), the slot gx values (1 per slot), the pair-rule records prec1 (kPr1
// per owned pair) and prec2 (kPr2 per owned pair), each part starting on a
// 32-byte boundary.
inline size_t round8(size_t v) { return (v + 7) / 8 * 8; }
inline size_t pbuf_gx_offset(long long n_slots) { return round8(4 * (size_t)n_slots); }
inline size_t pbuf_prec1_offset(long long n_slots) {
  return pbuf_gx_offset(n_slots) + round8((size_t)n_slots);
}
inline size_t prec2_offset(long long n_own) { return round8((size_t)kPr1 * (size_t)n_own); }
inline size_t pbuf_values(long long n_slots, long long n_own) {
  return pbuf_prec1_offset(n_slots) + prec2_offset(n_own) + (size_t)kPr2 * (size_t)n_own;
}
template <class R> inline bool has_undirected(const EvalArgs<R> &a) {
  return a.rev && a.pbuf && a.pgx && a.prec1 && a.prec2 && a.slot_own;
}

// Times every pass-1 and pass-2 variant on this input (reps launches each,
// synchronising st) and returns the fastest of each.  Every variant computes
// bitwise identical results; only the launch shape differs.
template <class R>
cudaError_t autotune_passes(const EvalArgs<R> &a, cudaStream_t st, int reps, int *best1,
                            int *best2);

// Deterministic FP64 totals over real sites: out[0] = sum V0, out[1] = sum S0,
// out[2] = sum |R_q|^2 + R_sigma^2 (active sites), out[3] = sum R_x^2.  Two
// launches; part is device scratch of kTotParts * 4 doubles per system.
constexpr int kTotParts = 64, kTotThreads = 256;
cudaError_t launch_totals(int n_real, const double *V0, const double *S0,
                          const double *Rq, const double *Rs, const double *Rx,
                          double *out, double *part, cudaStream_t st);

// Totals of each system of a batch: out[4k..4k+3] as launch_totals over the
// real sites [seg[k], seg[k+1]), bitwise equal to that system's own totals.
cudaError_t launch_seg_totals(int n_sys, const int *seg, const double *V0, const double *S0,
                              const double *Rq, const double *Rs, const double *Rx,
                              double *out, double *part, cudaStream_t st);

// Non-mean-field density rho_i = sum_j x_j rho_{s_j}(|q_i - q_j|)
// (density.cpp:44-104) for every real site.
// Mean-field stress W0 (9 per real site, row-major) from the moment
// records of a directed pass 1 (launch_pass1 with variants 0, 0).
template <class R>
cudaError_t launch_mf_stress(const EvalArgs<R> &a, double *W0, cudaStream_t st);
// Unweighted per-pair terms of the residual assembly from the moment records
// of a directed pass 1: self (5 per real site) = dV0_u/d(q_u, sigma_u, x_u),
// slot (5 per slot of the real sites' lists) = dV0_j/d(q_u, sigma_u, x_u).
template <class R>
cudaError_t launch_mf_pair_terms(const EvalArgs<R> &a, double *self, double *slot,
                                 cudaStream_t st);
cudaError_t launch_rho_nmf(int n_real, const double4 *pos, const double2 *xb,
                           const int *code, const int *offs, const int *idx,
                           SplineView<double> rho_mg, SplineView<double> rho_h,
                           double *out, cudaStream_t st);

}  // namespace btam
