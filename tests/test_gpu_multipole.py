"""The multipole rule (MULTIPOLE_INTEGRAL) on the device against the
reference built with it (tests/golden/multipole.npz, from
tests/golden/make_golden.py): rho-bar and V0 of every real site under
rule 1 (the reference's build flags: finite-difference Hessians) and rule
2 (analytic Hessians)."""
import os

import numpy as np
import pytest

import btam

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def load(name):
    return dict(np.load(os.path.join(GOLD, f"{name}.npz")))


def system_of(g):
    return {k: g[k] for k in ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell",
                              "periodic")}


@pytest.mark.parametrize("rule", [btam.MP_FD, btam.MP_ANALYTIC])
@pytest.mark.parametrize("name", ["sphere", "ortho_mgh"])
def test_multipole_against_reference(gpu_tables, name, rule):
    g, m = load(name), load("multipole")
    key = f"{name}_r{rule}_"
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    rho, V0, E = S.mf_eval_multipole(rule)
    # each term restates the reference's arithmetic; only the order of the
    # per-site sums differs (lanes of a warp)
    tol = 1e-12
    assert np.allclose(rho, m[key + "rho"], rtol=tol, atol=0)
    assert np.abs(V0 - m[key + "V0"]).max() <= tol * np.abs(m[key + "V0"]).max()
    assert abs(E - m[key + "V0"].sum()) <= tol * np.abs(m[key + "V0"]).sum()
    assert np.abs(S.last_S0 - m[key + "S0"]).max() <= tol * np.abs(m[key + "S0"]).max()
    # reproducible, and different from the degree-3 rule
    rho2, V02, E2 = S.mf_eval_multipole(rule)
    assert np.array_equal(rho, rho2) and np.array_equal(V0, V02) and E == E2
    assert np.abs(rho - g["rho"]).max() > 1e-6 * np.abs(g["rho"]).max()


@pytest.mark.parametrize("rule", [btam.MP_FD, btam.MP_ANALYTIC])
@pytest.mark.parametrize("name", ["sphere", "ortho_mgh"])
def test_multipole_residuals_against_reference(gpu_tables, name, rule):
    g, m = load(name), load("multipole")
    key = f"{name}_r{rule}_"
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    Rq, Rs, Rx = S.mf_residuals_multipole(rule)
    us = m[key + "res_sites"]
    # the reference's terms restated term by term; the per-site sums run in
    # another order, and the finite differences amplify that rounding
    for a, b in ((Rq[us], m[key + "Rq"]), (Rs[us], m[key + "Rs"]), (Rx[us], m[key + "Rx"])):
        assert np.abs(a - b).max() <= 1e-11 * max(1.0, np.abs(b).max())
    Rq2, Rs2, Rx2 = S.mf_residuals_multipole(rule)
    assert np.array_equal(Rq, Rq2) and np.array_equal(Rs, Rs2) and np.array_equal(Rx, Rx2)


@pytest.mark.parametrize("rule", [btam.MP_FD, btam.MP_ANALYTIC])
@pytest.mark.parametrize("name", ["sphere", "ortho_mgh"])
def test_multipole_stress_against_reference(gpu_tables, name, rule):
    """evaluate_DV0_i_dF_bulk_MgHx under the rule, q0 = q."""
    g, m = load(name), load("multipole")
    b = m[f"{name}_r{rule}_W0"]
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    W, tot = S.mf_stress_multipole(rule)
    assert np.abs(W - b).max() <= 1e-11 * max(1.0, np.abs(b).max())
    assert np.abs(tot - b.sum(axis=0)).max() <= 1e-11 * max(1.0, np.abs(b).sum(axis=0).max())


@pytest.mark.parametrize("rule", [btam.MP_FD, btam.MP_ANALYTIC])
@pytest.mark.parametrize("name", ["sphere", "ortho_mgh"])
def test_multipole_hessian_against_reference(gpu_tables, name, rule):
    """evaluate_D2V0_i_Dmeanq2_u_MgHx built with the rule, summed over
    i in {u} U N(u)."""
    g, m = load(name), load("multipole")
    b = m[f"{name}_r{rule}_H0"]
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    H = S.mf_hessian_multipole(rule)
    assert np.abs(H - b).max() <= 1e-9 * max(1.0, np.abs(b).max())
    assert np.array_equal(H, np.transpose(H, (0, 2, 1)))


def test_multipole_rejects_unknown_rule(gpu_tables):
    g = load("sphere")
    S = btam.System(gpu_tables, system_of(g))
    S.build_neighbors()
    for rule in (0, 3, -1):
        with pytest.raises(btam.BtamError):
            S.mf_eval_multipole(rule)
        with pytest.raises(btam.BtamError):
            S.mf_residuals_multipole(rule)
        with pytest.raises(btam.BtamError):
            S.mf_stress_multipole(rule)
        with pytest.raises(btam.BtamError):
            S.mf_hessian_multipole(rule)


def test_multipole_full_size_translation_invariance(gpu_tables):
    """Plain drop-in size (27,000 sites), rule 2: the per-site values stay
    finite and the multipole residual R_q sums to zero over the periodic
    cell (uniform beta; every term depends on differences of positions)."""
    from btam import lattice
    s = lattice.config2()
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    rho, V0, E = S.mf_eval_multipole(btam.MP_ANALYTIC)
    assert np.isfinite(V0).all() and np.isfinite(E)
    Rq, Rs, Rx = S.mf_residuals_multipole(btam.MP_ANALYTIC)
    assert np.isfinite(Rq).all() and np.isfinite(Rs).all() and np.isfinite(Rx).all()
    assert np.abs(Rq.sum(axis=0)).max() < 1e-8 * max(1.0, np.abs(Rq).max()) * len(Rq) ** 0.5


def test_multipole_sigma_derivative_by_differences(gpu_tables):
    """Rule 2 (analytic Hessians): R_sigma + 3 / (beta sigma) is the exact
    derivative of sum_i V0_i in sigma_u (uniform beta), checked by central
    differences of the device energy."""
    g = load("ortho_mgh")
    s = system_of(g)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    _, _, E0 = S.mf_eval_multipole(btam.MP_ANALYTIC)
    _, Rs, _ = S.mf_residuals_multipole(btam.MP_ANALYTIC)
    beta, sigma, x = s["beta"], s["sigma"], s["x"]
    assert np.ptp(beta) == 0.0
    h = 1e-5
    for u in np.flatnonzero(x >= 5e-4)[::37][:6]:
        sp, sm = sigma.copy(), sigma.copy()
        sp[u] += h
        sm[u] -= h
        S.set_state(sigma=sp)
        Ep = S.mf_eval_multipole(btam.MP_ANALYTIC)[2]
        S.set_state(sigma=sm)
        Em = S.mf_eval_multipole(btam.MP_ANALYTIC)[2]
        S.set_state(sigma=sigma)
        fd = (Ep - Em) / (2 * h)
        an = Rs[u] + 3.0 / (beta[u] * sigma[u])
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (u, fd, an)
