"""The reference's per-site plugin table (dmd_equations) served by
libbtam through include/btam_dmd_equations.hpp: a reference-style caller
(tests/compat/compat_probe.cpp) evaluates a system site by site and sums the
per-pair derivatives over i in {u} U N(u) (images included), as a residual
assembly would; the per-site values must equal the direct evaluation
through the C ABI to the bit, and the sums the assembled residuals within
1e-12.  The table is also driven one (u, i) pair at a time against the
reference's per-pair values (tests/golden/pairs.npz), and a state change
anywhere in N(i) must reach the value of (u, i)."""
import os
import subprocess

import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu
TABLES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "bt-am_b200", "data")


def write_system(path, s):
    n = len(s["x"])
    with open(path, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.ascontiguousarray(s["species"], np.int32).tobytes())
        for k in ("q", "sigma", "x", "beta", "gamma", "origin", "cell"):
            f.write(np.ascontiguousarray(s[k], np.float64).tobytes())
        f.write(np.ascontiguousarray(s["periodic"], np.int32).tobytes())


def test_plugin_table_matches_direct_evaluation(gpu_tables, tmp_path):
    import compat_build
    probe = compat_build.build_probe()
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.5, x_range=(0.0, 0.4),
                          sigma_range=(0.08, 0.15), jitter=0.02, seed=23)
    n = len(s["x"])
    inp, out = str(tmp_path / "sys.bin"), str(tmp_path / "out.bin")
    write_system(inp, s)
    r = subprocess.run([probe, TABLES, inp, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    v = np.frombuffer(raw[:8 * 8 * n], np.float64).reshape(n, 8)
    assert np.frombuffer(raw[8 * 8 * n:], np.int32)[0] == 0
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    d = S.evaluate(btam.FP64)
    assert np.array_equal(v[:, 0], d["rho"]) and np.array_equal(v[:, 1], d["V0"])
    assert np.array_equal(v[:, 2], d["S0"])
    # the caller's sums are the per-pair terms summed in list order
    selfv, slot = S.pair_terms(btam.FP64)
    offs, _ = S.neighbors()
    sums = selfv.copy()
    for u in range(n):
        for p in range(offs[u], offs[u + 1]):
            sums[u] += slot[p]
    assert np.array_equal(v[:, 3:8], sums)
    # and, beta being uniform here, the assembled residuals
    beta, sigma, x, gamma = s["beta"], s["sigma"], s["x"], s["gamma"]
    assert np.ptp(beta) == 0.0
    dsig = d["Rs"] + 3.0 / (beta * sigma)
    h = (s["species"] == 1) & (x >= 5e-4)
    dlogz = 3.0 / (2.0 * x[h]) + np.where(x[h] < 1.0, 1.0 / (1.0 - x[h]), 0.0)
    dx = d["Rx"][h] + dlogz / beta[h] + np.where(x[h] < 0.9999, gamma[h] / beta[h], 0.0)
    scale = max(1.0, np.abs(d["Rq"]).max(), np.abs(dsig).max(), np.abs(dx).max())
    assert np.abs(v[:, 3:6] - d["Rq"]).max() <= 1e-12 * scale
    assert np.abs(v[:, 6] - dsig).max() <= 1e-12 * scale
    assert np.abs(v[h, 7] - dx).max() <= 1e-12 * scale


@pytest.mark.parametrize("defines,rule", [
    (("MULTIPOLE_INTEGRAL", "NUMERICAL_DERIVATIVES=0"), btam.MP_FD),
    (("MULTIPOLE_INTEGRAL",), btam.MP_ANALYTIC)])
def test_plugin_table_multipole_build(gpu_tables, tmp_path, defines, rule):
    """A caller compiled with the reference's MULTIPOLE_INTEGRAL switch (and
    its NUMERICAL_DERIVATIVES, or without it) gets the multipole rule's
    values and derivatives."""
    import compat_build
    probe = compat_build.build_probe(defines)
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.5, x_range=(0.0, 0.4),
                          sigma_range=(0.08, 0.15), jitter=0.02, seed=29)
    n = len(s["x"])
    inp, out = str(tmp_path / "sys.bin"), str(tmp_path / "out.bin")
    write_system(inp, s)
    r = subprocess.run([probe, TABLES, inp, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    v = np.frombuffer(raw[:8 * 8 * n], np.float64).reshape(n, 8)
    assert np.frombuffer(raw[8 * 8 * n:], np.int32)[0] == 0
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    rho, V0, _ = S.mf_eval_multipole(rule)
    Rq, Rs, Rx = S.mf_residuals_multipole(rule)
    assert np.array_equal(v[:, 0], rho) and np.array_equal(v[:, 1], V0)
    assert np.array_equal(v[:, 2], S.last_S0)
    beta, sigma = s["beta"], s["sigma"]
    dsig = Rs + 3.0 / (beta * sigma)
    scale = max(1.0, np.abs(Rq).max(), np.abs(dsig).max())
    assert np.abs(v[:, 3:6] - Rq).max() <= 1e-12 * scale
    assert np.abs(v[:, 6] - dsig).max() <= 1e-12 * scale
    # and it is not the degree-3 rule
    assert np.abs(rho - S.evaluate(btam.FP64)["rho"]).max() > 1e-8


def test_plugin_table_point_forms_match_reference(gpu_tables, tmp_path):
    """The non-mean-field slots (evaluate_rho_i, evaluate_DV_i_Dq_j,
    evaluate_DV_i_DF) driven the way the reference's bulk residual drives
    them, and the mean-field stretch slot evaluate_DV0_i_DF, unstretched and
    at a stretch of the bound positions, against the reference's own values
    (tests/golden/point.npz)."""
    import compat_build
    probe = compat_build.build_probe()
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    g = dict(np.load(os.path.join(gold, "ortho_mgh.npz")))
    p = dict(np.load(os.path.join(gold, "point.npz")))
    s = {k: g[k] for k in ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell",
                           "periodic")}
    n = len(s["x"])
    inp = str(tmp_path / "sys.bin")
    write_system(inp, s)
    vol = abs(np.linalg.det(s["cell"].reshape(3, 3)))
    for F, kr, kw in ((np.ones(3), "ortho_mgh_rho", "ortho_mgh_W"),
                      (p["stretch"], "ortho_mgh_rho_s", "ortho_mgh_W_s")):
        out = str(tmp_path / "out.bin")
        r = subprocess.run([probe, TABLES, inp, out, "pt"] + [repr(float(f)) for f in F],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        raw = open(out, "rb").read()
        v = np.frombuffer(raw[:8 * 40 * n], np.float64).reshape(n, 40)
        Y = np.frombuffer(raw[8 * 40 * n:8 * 40 * n + 24], np.float64)
        assert np.frombuffer(raw[8 * 40 * n + 24:], np.int32)[0] == 0
        assert np.max(np.abs(v[:, 0] - p[kr])) <= 1e-12 * np.abs(p[kr]).max()
        W = v[:, 4:13].reshape(n, 3, 3)
        W0, kw0 = v[:, 13:22].reshape(n, 3, 3), kw.replace("_W", "_W0")
        assert np.max(np.abs(W0 - p[kw0])) <= 1e-10 * max(1.0, np.abs(p[kw0]).max())
        assert np.max(np.abs(W - p[kw])) <= 1e-10 * max(1.0, np.abs(p[kw]).max())
        Yref = np.array([p[kw][:, a, a].sum() for a in range(3)]) / vol
        assert np.max(np.abs(Y - Yref)) <= 1e-10 * max(1.0, np.abs(Yref).max())
        if F[0] == 1.0:
            Fq = p["ortho_mgh_Fq"]
            assert np.max(np.abs(v[:, 1:4] - Fq)) <= 1e-10 * max(1.0, np.abs(Fq).max())
            H = p["ortho_mgh_H"]
            assert np.max(np.abs(v[:, 22:31].reshape(n, 3, 3) - H)) <= 1e-9 * max(
                1.0, np.abs(H).max())
            H0 = p["ortho_mgh_H0"]
            assert np.max(np.abs(v[:, 31:].reshape(n, 3, 3) - H0)) <= 1e-9 * max(
                1.0, np.abs(H0).max())


PAIR_SYSTEMS = ["sphere", "x5cube", "ortho_mgh", "config1", "hot_cell"]


def pairs_golden(name):
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    p = dict(np.load(os.path.join(gold, "pairs.npz")))
    if name == "hot_cell":
        g = {k[len("hot_cell_"):]: v for k, v in p.items() if k.startswith("hot_cell_")}
    else:
        g = dict(np.load(os.path.join(gold, f"{name}.npz")))
    return p, g


def run_pairs(probe, tmp_path, s, ui):
    inp, out, pf = (str(tmp_path / "sys.bin"), str(tmp_path / "out.bin"),
                    str(tmp_path / "pairs.bin"))
    write_system(inp, s)
    with open(pf, "wb") as f:
        f.write(np.int32(len(ui)).tobytes())
        f.write(np.ascontiguousarray(ui, np.int32).tobytes())
    r = subprocess.run([probe, TABLES, inp, out, "pairs", pf], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    assert np.frombuffer(raw[8 * 30 * len(ui):], np.int32)[0] == 0
    return np.frombuffer(raw[:8 * 30 * len(ui)], np.float64).reshape(len(ui), 30)


@pytest.mark.parametrize("name", PAIR_SYSTEMS)
def test_plugin_table_pair_by_pair(gpu_tables, tmp_path, name):
    """Every derivative slot called one (u, i) pair at a time gives the
    reference's per-pair value: for i = u, for every neighbour i as u's list
    names it (images included) and for the pair as the reference evaluates
    it (u's image in i's list, i real).  hot_cell has a different
    temperature on every site."""
    import compat_build
    probe = compat_build.build_probe()
    p, g = pairs_golden(name)
    s = {k: g[k] for k in ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell",
                           "periodic")}
    us, k, entry = p[f"{name}_us"], p[f"{name}_k"], p[f"{name}_entry"]
    u = us[k]
    i = np.where(entry < 0, u, g["idx"][np.maximum(entry, 0)])
    tol = lambda a, b, t: np.max(np.abs(a - b)) <= t * max(1.0, np.abs(b).max())
    for ui in (np.column_stack([u, i]), np.column_stack([p[f"{name}_uu"], p[f"{name}_oo"]])):
        v = run_pairs(probe, tmp_path, s, ui)
        assert tol(v[:, :4], p[f"{name}_g4"], 1e-10)
        assert tol(v[:, 4], p[f"{name}_gx"], 1e-10)
        assert np.array_equal(v[:, 5:8], v[:, :3]) and np.array_equal(v[:, 8], v[:, 3])
        assert tol(v[:, 9:12], p[f"{name}_pt_g3"], 1e-10)
        assert tol(v[:, 12:21], p[f"{name}_pt_h9"].reshape(-1, 9), 1e-9)
        assert tol(v[:, 21:30], p[f"{name}_mf_h9"].reshape(-1, 9), 1e-9)


def test_plugin_table_sees_second_shell_changes(gpu_tables, tmp_path):
    """The value of (u, i) depends on every neighbour of i.  Moving a site j
    that neighbours i but not u (the second shell of u) must change it, and
    the new value must be that of the moved state."""
    import compat_build
    probe = compat_build.build_probe()
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.5, x_range=(0.05, 0.4),
                          sigma_range=(0.08, 0.15), jitter=0.02, seed=31)
    n = len(s["x"])
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    offs, idx = S.neighbors()
    owner = np.concatenate([np.arange(n), S.ghosts()[1]])
    lists = [set(owner[idx[offs[a]:offs[a + 1]]]) for a in range(n)]
    u = 0
    i = next(int(j) for j in idx[offs[u]:offs[u + 1]] if j < n)
    j = next(int(t) for t in sorted(lists[i] - lists[u] - {u, i}) if t < n)
    inp, out = str(tmp_path / "sys.bin"), str(tmp_path / "out.bin")
    write_system(inp, s)
    r = subprocess.run([probe, TABLES, inp, out, "perturb", str(u), str(i), str(j), "0.01"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    v = np.frombuffer(raw[:80], np.float64).reshape(2, 5)
    assert np.frombuffer(raw[80:], np.int32)[0] == 0
    slot_ui = offs[u] + list(idx[offs[u]:offs[u + 1]]).index(i)
    before = S.pair_terms(btam.FP64)[1][slot_ui]
    q = s["q"].copy()
    q[j, 0] += 0.01
    S.set_state(q=q)
    after = S.pair_terms(btam.FP64)[1][slot_ui]
    assert np.array_equal(v[0], before) and np.array_equal(v[1], after)
    assert np.abs(after - before).max() > 1e-8
