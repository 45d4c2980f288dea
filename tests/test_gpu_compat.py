"""The reference's per-site plugin table (dmd_equations) served by
libbtam through include/btam_dmd_equations.hpp: a reference-style caller
(tests/compat/compat_probe.cpp) evaluates a system site by site and sums the
pair derivatives over i in {u} U N(u), as a residual assembly would; the
per-site values and the assembled derivatives must equal the direct
evaluation through the C ABI, to the bit for the values and within 1e-12
for the derivatives the adapter rebuilds from the residuals."""
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
    assert np.array_equal(v[:, 2], d["S0"]) and np.array_equal(v[:, 3:6], d["Rq"])
    beta, sigma, x, gamma = s["beta"], s["sigma"], s["x"], s["gamma"]
    dsig = d["Rs"] + 3.0 / (beta * sigma)
    h = (s["species"] == 1) & (x >= 5e-4)
    dlogz = 3.0 / (2.0 * x[h]) + np.where(x[h] < 1.0, 1.0 / (1.0 - x[h]), 0.0)
    dx = np.zeros(n)
    dx[h] = d["Rx"][h] + dlogz / beta[h] + np.where(x[h] < 0.9999, gamma[h] / beta[h], 0.0)
    scale = max(1.0, np.abs(dsig).max(), np.abs(dx).max())
    assert np.abs(v[:, 6] - dsig).max() <= 1e-12 * scale
    assert np.abs(v[:, 7] - dx).max() <= 1e-12 * scale


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
    assert np.array_equal(v[:, 2], S.last_S0) and np.array_equal(v[:, 3:6], Rq)
    beta, sigma = s["beta"], s["sigma"]
    dsig = Rs + 3.0 / (beta * sigma)
    assert np.abs(v[:, 6] - dsig).max() <= 1e-12 * max(1.0, np.abs(dsig).max())
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
