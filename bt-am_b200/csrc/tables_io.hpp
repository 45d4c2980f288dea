// Host-side reader of the reference's ADP table files (plain C++).
//
// Format read by init_adp_MgHx (MgHx-ADP.cpp:366-501):
//   element file (adpmg.dat, adph.dat):  "mass factor r_cut",
//       "n dr" + n rows of 9 spline columns (rho), "n drho" + n rows (F),
//       then pair, u, w splines in the same "n dr" + rows form;
//   alloy file (adpmgh.dat):  "r_cut", then pair, u, w splines.
// Each row holds a, b, c, d, db, dc, dd, ddc, ddd; only a..d are kept
// because db = b, dc = 2c, dd = 3d (the derivative is formed from a..d).
#pragma once

#include <cstdio>
#include <string>
#include <vector>

namespace btam {

struct HostSpline {
  double dx = 0.0;
  int n = 0;
  std::vector<double> abcd;  // 4 per segment
};

struct HostTables {
  // index by TableId (adp_core.cuh)
  HostSpline t[13];
  double mass_mg = 0.0, mass_h = 0.0;
};

inline bool read_host_spline(FILE *f, HostSpline &s) {
  if (fscanf(f, "%d %lf", &s.n, &s.dx) != 2 || s.n <= 0 || !(s.dx > 0.0))
    return false;
  s.abcd.assign(4 * (size_t)s.n, 0.0);
  for (int i = 0; i < s.n; ++i) {
    double v[9];
    for (int c = 0; c < 9; ++c)
      if (fscanf(f, "%lf", &v[c]) != 1) return false;
    for (int c = 0; c < 4; ++c) s.abcd[4 * (size_t)i + c] = v[c];
  }
  return true;
}

// Returns 0 on success, 1 if a file is missing or malformed.
inline int load_host_tables(const std::string &dir, HostTables &T) {
  struct Spec {
    const char *file;
    bool alloy;
    int rho, emb, pair_kind;
  } specs[3] = {{"adpmg.dat", false, 0, 2, 0},
                {"adph.dat", false, 1, 3, 1},
                {"adpmgh.dat", true, -1, -1, 2}};
  for (const Spec &sp : specs) {
    FILE *f = fopen((dir + "/" + sp.file).c_str(), "r");
    if (!f) return 1;
    bool ok = true;
    if (!sp.alloy) {
      double mass, factor, rcut;
      ok = fscanf(f, "%lf %lf %lf", &mass, &factor, &rcut) == 3;
      if (sp.rho == 0) T.mass_mg = mass; else T.mass_h = mass;
      ok = ok && read_host_spline(f, T.t[sp.rho]) && read_host_spline(f, T.t[sp.emb]);
    } else {
      double rcut;
      ok = fscanf(f, "%lf", &rcut) == 1;
    }
    ok = ok && read_host_spline(f, T.t[4 + sp.pair_kind]) &&
         read_host_spline(f, T.t[7 + sp.pair_kind]) &&
         read_host_spline(f, T.t[10 + sp.pair_kind]);
    fclose(f);
    if (!ok) return 1;
  }
  return 0;
}

// Packs the radial tables into the kernels' per-segment records (layout at
// RadialView in adp_core.cuh): the uw block of pair kind pk at off_uw[pk] =
// off_uw[0] + 8 n pk, the pr block at off_pr[pk] = off_pr[0] + 8 n pk, all
// offsets multiples of 8 values.  Table ids: 0 rho_Mg, 1 rho_H,
// 4 + pk phi, 7 + pk u, 10 + pk w.  Returns false when the radial tables do
// not share one knot grid (then the records cannot serve them).
template <class R>
bool pack_radial(const HostTables &T, std::vector<R> &buf, size_t off_uw[3], size_t off_pr[3],
                 double &dx, int &n) {
  const int ids[11] = {0, 1, 4, 5, 6, 7, 8, 9, 10, 11, 12};
  n = T.t[0].n;
  dx = T.t[0].dx;
  for (int id : ids)
    if (T.t[id].n != n || T.t[id].dx != dx) return false;
  const size_t N = (size_t)n;
  size_t at = 0;
  for (int pk = 0; pk < 3; ++pk) {
    off_uw[pk] = at;
    at += 8 * N;
  }
  for (int pk = 0; pk < 3; ++pk) {
    off_pr[pk] = at;
    at += (pk == 2 ? 16 : 8) * N;
  }
  buf.assign(at, (R)0);
  auto put = [&](size_t dst, int id, size_t m) {
    for (int c = 0; c < 4; ++c) buf[dst + c] = (R)T.t[id].abcd[4 * m + c];
  };
  for (size_t m = 0; m < N; ++m)
    for (int pk = 0; pk < 3; ++pk) {
      put(off_uw[pk] + 8 * m, 7 + pk, m);
      put(off_uw[pk] + 8 * m + 4, 10 + pk, m);
      const size_t st = pk == 2 ? 16 : 8;
      put(off_pr[pk] + st * m, 4 + pk, m);
      if (pk == 2) {
        put(off_pr[pk] + st * m + 4, 0, m);
        put(off_pr[pk] + st * m + 8, 1, m);
      } else {
        put(off_pr[pk] + st * m + 4, pk, m);  // rho of the kind's species
      }
    }
  return true;
}

}  // namespace btam
