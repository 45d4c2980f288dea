// Test infrastructure only: the product's per-pair arithmetic
// (bt-am_b200/csrc/adp_core.cuh) compiled for the host and driven by plain
// sequential loops.  It lets the CPU test suite check the moment
// decomposition against the literal oracle without a GPU; the product path
// never calls it (the CUDA kernels are the product).
#include "../../bt-am_b200/csrc/adp_core.cuh"
#include "../../bt-am_b200/csrc/tables_io.hpp"

#include <array>
#include <cstring>
#include <vector>

using namespace btam;

namespace {
HostTables gT;
std::vector<Coef4<double>> gC64[13];
std::vector<Coef4<float>> gC32[13];

std::vector<double> gR64;
std::vector<float> gR32;
size_t gUW64[3], gPR64[3], gUW32[3], gPR32[3];
double gDx = 0.0;
int gN = 0;

template <class R> RadialView<R> radial(std::vector<R> &buf, const size_t *uw, const size_t *pr) {
  RadialView<R> v;
  v.uw = buf.data() + uw[0];
  v.pr = buf.data() + pr[0];
  v.dx = (R)gDx;
  v.inv_dx = (R)(1.0 / gDx);
  v.n = gN;
  return v;
}
template <class R> RadialView<R> rview();
template <> RadialView<double> rview<double>() { return radial(gR64, gUW64, gPR64); }
template <> RadialView<float> rview<float>() { return radial(gR32, gUW32, gPR32); }

template <class R> TablesView<R> view();
template <> TablesView<double> view<double>() {
  TablesView<double> v;
  for (int t = 0; t < 13; ++t)
    v.t[t] = SplineView<double>{gC64[t].data(), gT.t[t].dx, 1.0 / gT.t[t].dx, gT.t[t].n};
  return v;
}
template <> TablesView<float> view<float>() {
  TablesView<float> v;
  for (int t = 0; t < 13; ++t)
    v.t[t] = SplineView<float>{gC32[t].data(), (float)gT.t[t].dx,
                               (float)(1.0 / gT.t[t].dx), gT.t[t].n};
  return v;
}

template <class R>
void run(bool sym, int n_all, int n_real, const double *q, const double *sigma,
         const double *x, const int *code, const double *beta,
         const double *gamma, const int *owner, const int *offs,
         const int *idx, double *rho, double *V0, double *S0, double *selfx,
         double *Rq, double *Rs, double *Rx) {
  RadialView<R> T = rview<R>();
  SplineView<double> emb[2] = {view<double>().t[T_F_MG], view<double>().t[T_F_H]};
  std::vector<double> mom((size_t)n_real * kMomStride, 0.0);
  std::vector<R> momR((size_t)n_real * kMomStride, (R)0);
  std::vector<double> sx(n_real, 0.0);
  // undirected form: reverse slots, owned pairs (u < owner of j, or no
  // reverse slot) with one pair-rule record each, and each slot's owned pair
  // and direction (2 t + 0: the owned slot, 2 t + 1: its reverse)
  std::vector<int> rev(offs[n_real], -1), slot_own(offs[n_real], -1);
  std::vector<int> own_p;
  std::vector<std::array<R, kPrRec>> prec;
  if (sym) {
    for (int u = 0; u < n_real; ++u)
      for (int p = offs[u]; p < offs[u + 1]; ++p) {
        int o = owner[idx[p]];
        for (int t = offs[o]; t < offs[o + 1]; ++t)
          if (owner[idx[t]] == u) rev[p] = t;
      }
    for (int u = 0; u < n_real; ++u)
      for (int p = offs[u]; p < offs[u + 1]; ++p) {
        int j = idx[p], o = owner[j];
        if (!(u < o || rev[p] < 0)) continue;
        const int t = (int)own_p.size();
        own_p.push_back(p);
        slot_own[p] = 2 * t;
        if (rev[p] >= 0) slot_own[rev[p]] = 2 * t + 1;
        std::array<R, kPrRec> rec{};
        if (!(x[u] < kMinOcc) && !(x[j] < kMinOcc)) {
          V3<R> r0 = mk3<R>((R)(q[3 * u] - q[3 * j]), (R)(q[3 * u + 1] - q[3 * j + 1]),
                            (R)(q[3 * u + 2] - q[3 * j + 2]));
          R r[kPrRec];
          pair_rule_record<R>(T, r0, (R)sigma[u], (R)sigma[j], (R)x[u], (R)x[j], code[u],
                              code[j], r);
          for (int c = 0; c < kPrRec; ++c) rec[c] = r[c];
        }
        prec.push_back(rec);
      }
  }
  for (int i = 0; i < n_real; ++i) {
    rho[i] = V0[i] = S0[i] = selfx[i] = 0.0;
    if (x[i] < kMinOcc) continue;
    SiteSums S;
    memset(&S, 0, sizeof(S));
    for (int p = offs[i]; p < offs[i + 1]; ++p) {
      int j = idx[p];
      if (x[j] < kMinOcc) continue;
      V3<R> r0 = mk3<R>((R)(q[3 * i] - q[3 * j]), (R)(q[3 * i + 1] - q[3 * j + 1]),
                        (R)(q[3 * i + 2] - q[3 * j + 2]));
      R acc[kP1PartI], acc2[kP1PartII];
      for (int c = 0; c < kP1PartI; ++c) acc[c] = (R)0;
      for (int c = 0; c < kP1PartII; ++c) acc2[c] = (R)0;
      if (sym) {
        const std::array<R, kPrRec> &pr = prec[slot_own[p] >> 1];
        const R X = (R)x[i] * (R)x[j];
        acc[kP1Rho] = (R)x[j] * pr[(slot_own[p] & 1) ? 0 : 1];
        acc[kP1Epair] = (R)0.5 * X * pr[2];
        acc[kP1Ediag] = X * X * pr[3];
      } else {
        R rj, ep, ed;
        pass1_pair_rule<R>(T, r0, (R)sigma[i], (R)sigma[j], (R)x[i], (R)x[j], code[i], code[j],
                           rj, nullptr, ep, ed);
        acc[kP1Rho] = rj; acc[kP1Epair] = ep; acc[kP1Ediag] = ed;
      }
      const R X = (R)x[i] * (R)x[j];
      const int pk = pair_kind(code[i], code[j]);
      pass1_pair_part1<R>(T, r0, (R)sigma[j], X, pk, acc);
      pass1_pair_part2<R>(T, r0, (R)sigma[i], X, pk, acc2);
      double *sd = reinterpret_cast<double *>(&S);
      for (int v = 0; v < kP1Gd; ++v)
        if (v != kP1Sself) sd[p1_site_slot(v)] += (double)acc[v];
      for (int t = 0; t < 1 + 54; ++t) sd[p1_site_slot(p1_part2_value(t))] += (double)acc2[t];
    }
    SiteResult res;
    double mass = code[i] == 1 ? gT.mass_h : gT.mass_mg;
    site_epilogue(S, emb[code[i]], x[i], code[i], beta[i], gamma[i], sigma[i],
                  mass, res, mom.data() + (size_t)i * kMomStride);
    rho[i] = res.rho; V0[i] = res.V0; S0[i] = res.S0; selfx[i] = res.selfx;
    sx[i] = res.selfx;
  }
  for (size_t k = 0; k < mom.size(); ++k) momR[k] = (R)mom[k];
  if (sym) {
    // undirected pairs: each owned slot (u < owner of j) gives both
    // directions; slot values are summed per site in slot order
    std::vector<Pass2Out<R>> buf(offs[n_real]);
    for (auto &b : buf) b = Pass2Out<R>{};
    for (int u = 0; u < n_real; ++u)
      for (int p = offs[u]; p < offs[u + 1]; ++p) {
        int j = idx[p], o = owner[j];
        if (!(u < o || rev[p] < 0) || x[u] < kMinOcc || x[j] < kMinOcc) continue;
        const MomRec<R, false> mu(momR.data() + (size_t)u * kMomStride);
        const MomRec<R, false> mj(momR.data() + (size_t)o * kMomStride);
        V3<R> r0 = mk3<R>((R)(q[3 * u] - q[3 * j]), (R)(q[3 * u + 1] - q[3 * j + 1]),
                          (R)(q[3 * u + 2] - q[3 * j + 2]));
        Pass2Out<R> ou{}, oj{};
        R pr[kPrRec];
        for (int c = 0; c < kPrRec; ++c) pr[c] = prec[slot_own[p] >> 1][c];
        pass2_pair_sym<R>(T, r0, (R)sigma[u], (R)sigma[j], (R)x[u], (R)x[j], code[u], code[j],
                          mu.scalar(0), mu.scalar(1), mj.scalar(0), mj.scalar(1),
                          (R)(beta[o] / beta[u]),
                          (R)(beta[u] / beta[o]), mu, mj, pr, ou, oj);
        buf[p] = ou;
        if (rev[p] >= 0) buf[rev[p]] = oj;
      }
    for (int u = 0; u < n_real; ++u) {
      Rq[3 * u] = Rq[3 * u + 1] = Rq[3 * u + 2] = 0.0;
      Rs[u] = Rx[u] = 0.0;
      if (x[u] < kMinOcc) continue;
      double gq[3] = {0, 0, 0}, gs = 0, gx = 0;
      for (int p = offs[u]; p < offs[u + 1]; ++p) {
        for (int k = 0; k < 3; ++k) gq[k] += buf[p].gq[k];
        gs += buf[p].gs;
        gx += buf[p].gx;
      }
      residual_epilogue(sigma[u], x[u], code[u], beta[u], gamma[u], sx[u], gs, gx);
      for (int k = 0; k < 3; ++k) Rq[3 * u + k] = gq[k];
      Rs[u] = gs;
      Rx[u] = gx;
    }
    return;
  }
  for (int u = 0; u < n_real; ++u) {
    Rq[3 * u] = Rq[3 * u + 1] = Rq[3 * u + 2] = 0.0;
    Rs[u] = Rx[u] = 0.0;
    if (x[u] < kMinOcc) continue;
    const MomRec<R, false> mu(momR.data() + (size_t)u * kMomStride);
    double gq[3] = {0, 0, 0}, gs = 0, gx = 0;
    for (int p = offs[u]; p < offs[u + 1]; ++p) {
      int j = idx[p];
      if (x[j] < kMinOcc) continue;
      int o = owner[j];
      const MomRec<R, false> mj(momR.data() + (size_t)o * kMomStride);
      V3<R> r0 = mk3<R>((R)(q[3 * u] - q[3 * j]), (R)(q[3 * u + 1] - q[3 * j + 1]),
                        (R)(q[3 * u + 2] - q[3 * j + 2]));
      Pass2Out<R> out{};
      pass2_pair<R>(T, r0, (R)sigma[u], (R)sigma[j], (R)x[u], (R)x[j], code[u],
                    code[j], mu.scalar(0), mj.scalar(0), mj.scalar(1), (R)(beta[o] / beta[u]),
                    mu, mj, out);
      for (int k = 0; k < 3; ++k) gq[k] += out.gq[k];
      gs += out.gs;
      gx += out.gx;
    }
    residual_epilogue(sigma[u], x[u], code[u], beta[u], gamma[u], sx[u], gs, gx);
    for (int k = 0; k < 3; ++k) Rq[3 * u + k] = gq[k];
    Rs[u] = gs;
    Rx[u] = gx;
  }
}
}  // namespace

extern "C" {
int hm_load_tables(const char *dir) {
  if (load_host_tables(dir, gT)) return 1;
  for (int t = 0; t < 13; ++t) {
    gC64[t].resize(gT.t[t].n);
    gC32[t].resize(gT.t[t].n);
    for (int m = 0; m < gT.t[t].n; ++m) {
      const double *c = &gT.t[t].abcd[4 * (size_t)m];
      gC64[t][m] = Coef4<double>{c[0], c[1], c[2], c[3]};
      gC32[t][m] = Coef4<float>{(float)c[0], (float)c[1], (float)c[2], (float)c[3]};
    }
  }
  if (!pack_radial(gT, gR64, gUW64, gPR64, gDx, gN) ||
      !pack_radial(gT, gR32, gUW32, gPR32, gDx, gN))
    return 1;
  return 0;
}

void hm_eval(int fp32, int sym, int n_all, int n_real, const double *q, const double *sigma,
             const double *x, const int *code, const double *beta,
             const double *gamma, const int *owner, const int *offs,
             const int *idx, double *rho, double *V0, double *S0,
             double *selfx, double *Rq, double *Rs, double *Rx) {
  if (fp32)
    run<float>(sym != 0, n_all, n_real, q, sigma, x, code, beta, gamma, owner, offs, idx,
               rho, V0, S0, selfx, Rq, Rs, Rx);
  else
    run<double>(sym != 0, n_all, n_real, q, sigma, x, code, beta, gamma, owner, offs, idx,
                rho, V0, S0, selfx, Rq, Rs, Rx);
}
}
