// Test infrastructure only: the product's per-pair arithmetic
// (bt-am_b200/csrc/adp_core.cuh) compiled for the host and driven by plain
// sequential loops.  It lets the CPU test suite check the moment
// decomposition against the literal oracle without a GPU; the product path
// never calls it (the CUDA kernels are the product).
#include "../../bt-am_b200/csrc/adp_core.cuh"
#include "../../bt-am_b200/csrc/tables_io.hpp"

#include <cstring>
#include <vector>

using namespace btam;

namespace {
HostTables gT;
std::vector<Coef4<double>> gC64[13];
std::vector<Coef4<float>> gC32[13];

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
  TablesView<R> T = view<R>();
  SplineView<double> emb[2] = {view<double>().t[T_F_MG], view<double>().t[T_F_H]};
  std::vector<double> mom((size_t)n_real * kMomStride, 0.0);
  std::vector<R> momR((size_t)n_real * kMomStride, (R)0);
  std::vector<double> sx(n_real, 0.0);
  // undirected form: reverse slots, and the pair-rule sums of every slot from
  // its owned pair (both directions at once)
  std::vector<int> rev(offs[n_real], -1);
  std::vector<R> rec(3 * (size_t)offs[n_real], (R)0);
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
        if (!(u < o || rev[p] < 0) || x[u] < kMinOcc || x[j] < kMinOcc) continue;
        V3<R> r0 = mk3<R>((R)(q[3 * u] - q[3 * j]), (R)(q[3 * u + 1] - q[3 * j + 1]),
                          (R)(q[3 * u + 2] - q[3 * j + 2]));
        R rj, ri, ep, ed;
        pass1_pair_rule<R>(T, r0, (R)sigma[u], (R)sigma[j], (R)x[u], (R)x[j], code[u], code[j],
                           rj, &ri, ep, ed);
        rec[3 * p] = rj; rec[3 * p + 1] = ep; rec[3 * p + 2] = ed;
        if (rev[p] >= 0) {
          rec[3 * rev[p]] = ri; rec[3 * rev[p] + 1] = ep; rec[3 * rev[p] + 2] = ed;
        }
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
      Pass1A<R> a;
      memset(&a, 0, sizeof(a));
      if (sym) {
        a.rho = rec[3 * p]; a.epair = rec[3 * p + 1]; a.ediag = rec[3 * p + 2];
        pass1_pair_trip<R>(T, r0, (R)sigma[j], (R)x[i] * (R)x[j], pair_kind(code[i], code[j]), a);
      } else {
        pass1_pair_A<R>(T, r0, (R)sigma[i], (R)sigma[j], (R)x[i], (R)x[j], code[i], code[j], a);
      }
      S.rho += a.rho; S.epair += a.epair; S.ediag += a.ediag; S.cross += a.cross;
      for (int c = 0; c < 3; ++c) { S.g0a[c] += a.g0.a[c]; S.ha[c] += a.hsum.a[c]; }
      for (int c = 0; c < 6; ++c) { S.g0l[c] += a.g0.l[c]; S.hl[c] += a.hsum.l[c]; }
      R X = (R)(x[i] * x[j]);
      int pk = pair_kind(code[i], code[j]);
      for (int k = 0; k < 3; ++k)
        for (int sg = 0; sg < 2; ++sg) {
          Feat<R> gd{};
          R ss = 0;
          pass1_pair_B<R>(T, r0, (R)sigma[i], X, pk, k, sg, gd, ss);
          int d = 2 * k + sg;
          for (int c = 0; c < 3; ++c) S.gda[d][c] += gd.a[c];
          for (int c = 0; c < 6; ++c) S.gdl[d][c] += gd.l[c];
          S.sself += ss;
        }
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
        const R *mu = momR.data() + (size_t)u * kMomStride;
        const R *mj = momR.data() + (size_t)o * kMomStride;
        V3<R> r0 = mk3<R>((R)(q[3 * u] - q[3 * j]), (R)(q[3 * u + 1] - q[3 * j + 1]),
                          (R)(q[3 * u + 2] - q[3 * j + 2]));
        Pass2Out<R> ou{}, oj{};
        pass2_pair_sym<R>(T, r0, (R)sigma[u], (R)sigma[j], (R)x[u], (R)x[j], code[u], code[j],
                          mu[0], mu[1], mj[0], mj[1], (R)(beta[o] / beta[u]),
                          (R)(beta[u] / beta[o]), mu, mj, ou, oj);
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
    const R *mu = momR.data() + (size_t)u * kMomStride;
    double gq[3] = {0, 0, 0}, gs = 0, gx = 0;
    for (int p = offs[u]; p < offs[u + 1]; ++p) {
      int j = idx[p];
      if (x[j] < kMinOcc) continue;
      int o = owner[j];
      const R *mj = momR.data() + (size_t)o * kMomStride;
      V3<R> r0 = mk3<R>((R)(q[3 * u] - q[3 * j]), (R)(q[3 * u + 1] - q[3 * j + 1]),
                        (R)(q[3 * u + 2] - q[3 * j + 2]));
      Pass2Out<R> out{};
      pass2_pair<R>(T, r0, (R)sigma[u], (R)sigma[j], (R)x[u], (R)x[j], code[u],
                    code[j], mu[0], mj[0], mj[1], (R)(beta[o] / beta[u]), mu, mj, out);
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
