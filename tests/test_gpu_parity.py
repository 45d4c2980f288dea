"""CUDA path (through the C ABI) against the oracle and the golden fixtures.

Tolerances: neighbour lists and periodic images bit-exact; FP64 form 1e-10
relative per-site energy and 1e-10 (relative to the largest component)
residuals; FP32C form <= 1e-6 relative total energy, <= 1e-5 eV/A residual
components (R_x relative to its scale)."""
import os

import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["sphere", "x5cube", "ortho_mgh", "config1"]
KEYS = ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell", "periodic")


def load(name):
    return dict(np.load(os.path.join(GOLD, f"{name}.npz")))


def system_of(g):
    return {k: g[k] for k in KEYS}


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", NAMES)
def test_images_and_neighbors_bit_exact(gpu_tables, name):
    g = load(name)
    n = len(g["x"])
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors(all_sites=True)
    qg, og, ig = S.ghosts()
    assert np.array_equal(qg, g["q_all"][n:])
    assert np.array_equal(og, g["owner"][n:]) and np.array_equal(ig, g["image"][n:])
    offs, idx = S.neighbors()
    assert np.array_equal(offs, g["offs"]) and np.array_equal(idx, g["idx"])


# launch variants (pass 1, pass 2): directed (each site over its neighbours)
# and undirected (each pair once for both directions), full and persistent
# grids
VARIANTS = [(0, 0), (0, 16), (16, 16), (16 | 8 | 3, 16 | 8 | 2), (16 | 8 | 3, 16 | 4)]


@pytest.mark.parametrize("v", VARIANTS, ids=lambda v: f"v{v[0]}-{v[1]}")
@pytest.mark.parametrize("name", NAMES)
def test_fp64_against_golden(gpu_tables, name, v):
    g = load(name)
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    S.set_variants(btam.FP64, *v)
    out = S.evaluate(btam.FP64)
    assert rel(out["rho"], g["rho"]) < 1e-12
    assert np.max(np.abs(out["V0"] - g["V0"]) / np.maximum(np.abs(g["V0"]), 1e-3)) < 1e-10
    assert rel(out["S0"], g["S0"]) < 1e-12
    us = g["res_sites"]
    for k in ("Rq", "Rs", "Rx"):
        assert np.max(np.abs(out[k][us] - g[k])) < 1e-10 * max(1.0, np.abs(g[k]).max()), k
    assert abs(out["totals"][0] - g["V0"].sum()) < 1e-10 * abs(g["V0"].sum())


@pytest.mark.parametrize("v", VARIANTS, ids=lambda v: f"v{v[0]}-{v[1]}")
@pytest.mark.parametrize("name", NAMES)
def test_fp32c_against_golden(gpu_tables, name, v):
    g = load(name)
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    S.set_variants(btam.FP32C, *v)
    out = S.evaluate(btam.FP32C)
    E0 = g["V0"].sum()
    assert abs(out["totals"][0] - E0) <= 1e-6 * abs(E0)
    us = g["res_sites"]
    assert np.max(np.abs(out["Rq"][us] - g["Rq"])) <= 1e-5
    assert np.max(np.abs(out["Rs"][us] - g["Rs"])) <= 1e-5
    assert np.max(np.abs(out["Rx"][us] - g["Rx"])) <= 1e-5 * max(1.0, np.abs(g["Rx"]).max())


def test_rho_nmf_and_splines(gpu_tables):
    g = load("ortho_mgh")
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    assert rel(S.rho_nmf(), g["rho_nmf"]) < 1e-13
    sp = load("splines")
    for t in range(13):
        v, d = gpu_tables.spline(t, sp[f"t{t}_r"])
        assert np.allclose(v, sp[f"t{t}_v"], rtol=1e-13, atol=1e-15)
        assert np.allclose(d, sp[f"t{t}_d"], rtol=1e-12, atol=1e-13)


def test_deterministic_and_state_update(gpu_tables, hostmodel, oracle):
    import pyoracle
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.4, x_range=(0.0, 0.5),
                          sigma_range=(0.07, 0.16), jitter=0.03, seed=8)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    a = S.evaluate(btam.FP64)
    b = S.evaluate(btam.FP64)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # new sigma and x through the C ABI; images follow their owners
    rng = np.random.default_rng(3)
    s2 = dict(s)
    s2["sigma"] = s["sigma"] * rng.uniform(0.9, 1.1, len(s["x"]))
    s2["x"] = np.where(s["species"] == 1, rng.uniform(0.0, 0.6, len(s["x"])), 1.0)
    S.set_state(sigma=s2["sigma"], x=s2["x"])
    out = S.evaluate(btam.FP64)
    full, n, owner, image = pyoracle.expand(s2, oracle)
    offs, idx = oracle.neighbors(full["q"])
    ref = hostmodel.evaluate(full, n, owner, offs, idx)
    for k in ("rho", "V0", "Rq", "Rs", "Rx"):
        assert rel(out[k], ref[k]) < 1e-11, k


def test_launch_variants(gpu_tables):
    """Every launch variant (block shape x full or persistent grid) runs the
    same per-site arithmetic in the same order: the grid never changes a bit;
    block shapes are separate compilations whose multiply-add contraction may
    differ, so they agree to rounding (FP64 1e-12 relative, FP32C within its
    stated tolerance); a pinned variant reproduces itself bitwise."""
    g = load("config1")
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    for prec, tol in ((btam.FP64, 1e-12), (btam.FP32C, 1e-6)):
        base = S.evaluate(prec)
        for shape1, shape2 in ([(v, v) for v in range(6)] +
                               [(0, 16 | v) for v in range(7)] +
                               [(16 | v, 16 | v) for v in range(6)] + [(16 | 5, 16 | 6)]):
            for pers in (0, 8):
                S.set_variants(prec, shape1 | pers, shape2 | pers)
                out = S.evaluate(prec)
                again = S.evaluate(prec)
                for k in out:
                    assert np.array_equal(out[k], again[k]), (prec, shape1, k)
                if pers:
                    for k in out:
                        assert np.array_equal(out[k], full[k]), (prec, shape1, "grid", k)
                else:
                    full = out
                for k in ("V0", "S0"):
                    assert rel(out[k], base[k]) < tol, (prec, shape1, k)
                for k in ("Rq", "Rs", "Rx"):
                    assert np.abs(out[k] - base[k]).max() < 10 * tol, (prec, shape1, k)
        v1, v2 = S.autotune(prec)
        assert (v1 & 7) < 6 and v1 < 32 and v2 < 32
        assert (v2 & 7) < (7 if v2 & 16 else 6)
    with pytest.raises(btam.BtamError):
        S.set_variants(btam.FP64, 6, 0)


def test_state_update_rejections(gpu_tables):
    """btam_system_set_state validates an update before it replaces the
    state: non-finite or non-positive values, a non-H site with
    0 < x < min_occupancy and a site outside a periodic cell are rejected
    with their codes, and the device keeps the previous state."""
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.5, x_range=(0.0, 0.3), seed=17)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    base = S.evaluate(btam.FP64)
    mg = np.flatnonzero(s["species"] == 12)[0]
    bad_q = s["q"].copy()
    bad_q[5, 1] = np.nan
    out_q = s["q"].copy()
    out_q[7, 0] = s["origin"][0] - 1.0
    bad_s = s["sigma"].copy()
    bad_s[3] = 0.0
    bad_x = s["x"].copy()
    bad_x[mg] = 1e-4
    for kw, code in ((dict(q=bad_q), 6), (dict(q=out_q), 14), (dict(sigma=bad_s), 6),
                     (dict(x=bad_x), 10)):
        with pytest.raises(btam.BtamError) as e:
            S.set_state(**kw)
        assert e.value.code == code, (kw.keys(), e.value.code)
        again = S.evaluate(btam.FP64)
        for k in ("V0", "Rq", "Rs", "Rx"):
            assert np.array_equal(again[k], base[k]), k


def test_eval_state_matches_set_state_then_eval(gpu_tables):
    """btam_mf_eval_state (one wait for the device) gives the bits of
    btam_system_set_state followed by btam_mf_eval, in both forms, and a
    rejected update returns the set_state code with the state kept."""
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.5, x_range=(0.0, 0.3), seed=17)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    rng = np.random.default_rng(4)
    cell = s["cell"].reshape(3, 3)
    lo, hi = s["origin"], s["origin"] + np.diag(cell)
    inside = np.all((s["q"] > lo + 0.05) & (s["q"] < hi - 0.05), axis=1)
    q2 = s["q"].copy()
    q2[inside] += rng.normal(0.0, 0.01, (int(inside.sum()), 3))
    sig2 = s["sigma"] * 1.05
    for prec in (btam.FP64, btam.FP32C):
        S.set_state(q=s["q"], sigma=s["sigma"], x=s["x"])
        S.set_state(q=q2, sigma=sig2)
        a = S.evaluate(prec)
        S.set_state(q=s["q"], sigma=s["sigma"], x=s["x"])
        b = S.evaluate_state(prec, q=q2, sigma=sig2)
        for k in a:
            assert np.array_equal(a[k], b[k]), (prec, k)
    base = S.evaluate(btam.FP64)
    bad_q = q2.copy()
    bad_q[5, 1] = np.nan
    with pytest.raises(btam.BtamError) as e:
        S.evaluate_state(btam.FP64, q=bad_q)
    assert e.value.code == 6
    again = S.evaluate(btam.FP64)
    for k in ("V0", "Rq", "Rs", "Rx"):
        assert np.array_equal(again[k], base[k]), k


def test_persistent_grid_bitwise_on_large_system(gpu_tables):
    """A system with more sites and pairs than one wave of resident blocks:
    the persistent grid computes most sites and pairs in later trips of its
    loops, and every result must still equal the full grid's bitwise."""
    s = lattice.supercell(12, 8, 8, ortho=True, h_fraction=0.5, x_range=(0.0, 0.4),
                          sigma_range=(0.08, 0.15), jitter=0.02, seed=41)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    for prec in (btam.FP64, btam.FP32C):
        for v1, v2 in [(0, 0), (1, 1), (3, 4), (2, 16), (4, 16 | 3), (0, 16 | 1), (16, 16),
                       (16 | 3, 16 | 2)]:
            S.set_variants(prec, v1, v2)
            full = S.evaluate(prec)
            S.set_variants(prec, v1 | 8, v2 | 8)
            pers = S.evaluate(prec)
            for k in full:
                assert np.array_equal(full[k], pers[k]), (prec, v1, v2, k)


def test_error_codes(gpu_tables):
    s = lattice.supercell(3, 2, 3, ortho=True, with_tetra=False)
    with pytest.raises(btam.BtamError) as e:
        btam.System(gpu_tables, s)  # periodic cell thinner than 2 rc
    assert e.value.code == 5
    s = lattice.cluster("sphere", 6.0, seed=1)
    bad = dict(s, species=np.where(s["species"] == 1, 2, s["species"]).astype(np.int32))
    with pytest.raises(btam.BtamError) as e:
        btam.System(gpu_tables, bad)
    assert e.value.code == 11
    bad = dict(s, x=np.where(s["species"] == 12, 1e-4, s["x"]))
    with pytest.raises(btam.BtamError) as e:
        btam.System(gpu_tables, bad)
    assert e.value.code == 10
    S = btam.System(gpu_tables, s)
    with pytest.raises(btam.BtamError) as e:
        S.evaluate()
    assert e.value.code == 13
    # an isolated site has no neighbours (Neighbors.cpp:106-113)
    iso = dict(s)
    iso["q"] = np.vstack([s["q"], [[60.0, 60.0, 60.0]]])
    for k in ("sigma", "x", "beta", "gamma"):
        iso[k] = np.append(s[k], s[k][0])
    iso["species"] = np.append(s["species"], 12).astype(np.int32)
    iso["cell"] = np.diag([80.0, 80.0, 80.0])
    iso["origin"] = np.array([-20.0, -20.0, -20.0])
    S = btam.System(gpu_tables, iso)
    with pytest.raises(btam.BtamError) as e:
        S.build_neighbors()
    assert e.value.code == 4
    # more than maxneigh = 250 neighbours (Neighbors.cpp:96-104)
    rng = np.random.default_rng(0)
    m = 300
    dense = dict(q=rng.uniform(-2.0, 2.0, (m, 3)), sigma=np.full(m, 0.1), x=np.ones(m),
                 species=np.full(m, 12, np.int32), beta=np.full(m, 38.68),
                 gamma=np.zeros(m), origin=np.full(3, -3.0), cell=np.diag([6.0] * 3),
                 periodic=np.zeros(3, np.int32))
    S = btam.System(gpu_tables, dense)
    with pytest.raises(btam.BtamError) as e:
        S.build_neighbors()
    assert e.value.code == 3


def test_full_size_config2(gpu_tables, oracle):
    """Plain drop-in size (9000 Mg + 18000 tetrahedral sites): sampled literal
    residuals, FP64 vs FP32C agreement, translation invariance and a
    finite-difference check of dE/dq."""
    import pyoracle
    s = lattice.config2()
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    a = S.evaluate(btam.FP64)
    b = S.evaluate(btam.FP32C)
    E64, E32 = a["totals"][0], b["totals"][0]
    assert abs(E32 - E64) <= 1e-6 * abs(E64)
    assert np.max(np.abs(b["Rq"] - a["Rq"])) <= 1e-5
    assert np.max(np.abs(b["Rs"] - a["Rs"])) <= 1e-5
    assert np.abs(a["Rq"].sum(axis=0)).max() < 1e-8
    sites = np.array([0, 17, 4500, 9000 + 3, 9000 + 1234, 26999], np.int32)
    lit = pyoracle.sampled_residuals(s, oracle, sites)
    assert rel(a["V0"][sites], lit["V0"]) < 1e-10
    for k in ("Rq", "Rs", "Rx"):
        assert np.max(np.abs(a[k][sites] - lit[k])) < 1e-10 * max(1.0, np.abs(lit[k]).max()), k
    # dE/dq by central differences (beta uniform, so R_q is the energy gradient)
    h = 1e-4
    frac = s["q"] @ np.linalg.inv(s["cell"])
    inside = np.all((frac > 0.05) & (frac < 0.95), axis=1) & (s["x"] >= 5e-4)
    picks = [np.flatnonzero(inside & (s["species"] == sp))[3] for sp in (12, 1)]
    for site, ax in ((picks[0], 0), (picks[1], 2)):
        E = []
        for sgn in (1, -1):
            q = s["q"].copy()
            q[site, ax] += sgn * h
            S.set_state(q=q)
            E.append(S.evaluate(btam.FP64)["totals"][0])
        S.set_state(q=s["q"])
        assert abs((E[0] - E[1]) / (2 * h) - a["Rq"][site, ax]) < 1e-5


def test_full_size_config3_nanowire(gpu_tables, oracle):
    """Precision workload (hcp Mg nanowire R = 30 A, 20 cells, periodic along
    the axis only, 38 040 sites with free surfaces): the FP32C form against
    the FP64 form at the form's stated tolerance on every result, the FP64
    form against sampled literal residuals of the oracle, and translation
    invariance (T is uniform, so sum_u R_q(u) is the gradient of the total
    energy under a rigid shift)."""
    import pyoracle
    s = lattice.config3()
    n = len(s["x"])
    assert n == 38040
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    a = S.evaluate(btam.FP64)
    b = S.evaluate(btam.FP32C)
    E64, E32 = a["totals"][0], b["totals"][0]
    assert abs(E32 - E64) <= 1e-6 * abs(E64)
    assert np.max(np.abs(b["V0"] - a["V0"])) <= 1e-5
    assert np.max(np.abs(b["Rq"] - a["Rq"])) <= 1e-5
    assert np.max(np.abs(b["Rs"] - a["Rs"])) <= 1e-5
    assert np.max(np.abs(b["Rx"] - a["Rx"])) <= 1e-5 * max(1.0, np.abs(a["Rx"]).max())
    assert np.abs(a["Rq"].sum(axis=0)).max() < 1e-8
    # surface and core sites of both species
    r = np.hypot(s["q"][:, 0] - s["q"][:, 0].mean(), s["q"][:, 1] - s["q"][:, 1].mean())
    picks = []
    for sp in (12, 1):
        m = s["species"] == sp
        picks += [np.flatnonzero(m & (r < 10.0))[0], np.flatnonzero(m & (r > 27.0))[0],
                  np.flatnonzero(m & (r > 27.0))[-1]]
    sites = np.array(sorted(set(map(int, picks))), np.int32)
    lit = pyoracle.sampled_residuals(s, oracle, sites)
    assert rel(a["V0"][sites], lit["V0"]) < 1e-10
    for k in ("Rq", "Rs", "Rx"):
        assert np.max(np.abs(a[k][sites] - lit[k])) < 1e-10 * max(1.0, np.abs(lit[k]).max()), k
