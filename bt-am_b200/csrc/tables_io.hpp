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

}  // namespace btam
