"""Per-pair terms on the device against the reference's per-pair functions.

The reference's plugin slots return one term per (u, i) call:
evaluate_DV0_i_Dq_u / _Dxi_u (MgHx-mf-V-bulk.cpp:1823-2325),
evaluate_DV_i_Dq_u (147-330), evaluate_D2V_i_Dq2_u (333-528) and
evaluate_D2V0_i_Dmeanq2_u (1366-1600).  tests/golden/pairs.npz holds the
reference's values for the self entry and every list entry of sampled sites
(tests/golden/make_golden.py), including a cell whose sites carry different
temperatures.  Tolerances: FP64 1e-10 of max(1, the largest golden
component) for gradients, 1e-9 for Hessian blocks (the degree-3 Hessian's
tolerance elsewhere), FP32C 1e-5."""
import os

import numpy as np
import pytest

import btam

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
SYSTEMS = ["sphere", "x5cube", "ortho_mgh", "config1", "hot_cell"]
KEYS = ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell", "periodic")


def load(name):
    p = dict(np.load(os.path.join(GOLD, "pairs.npz")))
    if name == "hot_cell":
        g = {k[len("hot_cell_"):]: v for k, v in p.items() if k.startswith("hot_cell_")}
    else:
        g = dict(np.load(os.path.join(GOLD, f"{name}.npz")))
    return p, g


def built(gpu_tables, g):
    S = btam.System(gpu_tables, {k: g[k] for k in KEYS})
    S.build_neighbors()
    n = len(g["x"])
    offs, idx = S.neighbors()
    # the real sites' lists are the fixture's (bit-exact neighbour lists)
    assert np.array_equal(offs, g["offs"][:n + 1])
    assert np.array_equal(idx, g["idx"][:offs[n]])
    return S


def device_rows(p, name, selfv, slot):
    """The device value for every golden row: the site's self entry or the
    list entry the row names."""
    us, k, entry = p[f"{name}_us"], p[f"{name}_k"], p[f"{name}_entry"]
    return np.where((entry < 0)[:, None], selfv[us[k]], slot[np.maximum(entry, 0)])


def close(a, b, tol):
    return np.max(np.abs(a - b)) <= tol * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("name", SYSTEMS)
def test_mean_field_pair_terms(gpu_tables, name):
    p, g = load(name)
    S = built(gpu_tables, g)
    gold = np.column_stack([p[f"{name}_g4"], p[f"{name}_gx"]])
    for prec, tol in ((btam.FP64, 1e-10), (btam.FP32C, 1e-5)):
        selfv, slot = S.pair_terms(prec)
        dev = device_rows(p, name, selfv, slot)
        assert close(dev[:, :4], gold[:, :4], tol), prec
        assert close(dev[:, 4], gold[:, 4], tol), prec


@pytest.mark.parametrize("name", SYSTEMS)
def test_point_and_hessian_pair_terms(gpu_tables, name):
    p, g = load(name)
    S = built(gpu_tables, g)
    g3, gp3, Hs, Hp = S.pt_pair_terms()
    ns = len(gp3)
    assert close(device_rows(p, name, g3, gp3), p[f"{name}_pt_g3"], 1e-10)
    H = device_rows(p, name, Hs.reshape(-1, 9), Hp.reshape(ns, 9))
    assert close(H, p[f"{name}_pt_h9"].reshape(-1, 9), 1e-9)
    Ms, Mp = S.mf_hessian_pairs()
    M = device_rows(p, name, Ms.reshape(-1, 9), Mp.reshape(ns, 9))
    assert close(M, p[f"{name}_mf_h9"].reshape(-1, 9), 1e-9)


@pytest.mark.parametrize("rule", [1, 2])
@pytest.mark.parametrize("name", ["sphere", "ortho_mgh"])
def test_multipole_pair_terms(gpu_tables, name, rule):
    p, g = load(name)
    S = built(gpu_tables, g)
    selfv, slot = S.pair_terms_multipole(rule)
    dev = device_rows(p, name, selfv, slot)
    gold = np.column_stack([p[f"{name}_mp{rule}_g4"], p[f"{name}_mp{rule}_gx"]])
    # the multipole tolerance of the assembled residuals (1e-11)
    assert close(dev, gold, 1e-11)
    Hs, Hp = S.mf_hessian_pairs(rule)
    H = device_rows(p, name, Hs.reshape(-1, 9), Hp.reshape(len(Hp), 9))
    assert close(H, p[f"{name}_mp{rule}_h9"].reshape(-1, 9), 1e-9)


def test_non_uniform_beta_sums(gpu_tables):
    """With temperatures that differ from site to site, a raw sum of the
    per-pair values over i equals the reference's raw sum, and the
    beta_i / beta_u weighted sum is the assembled residual."""
    p, g = load("hot_cell")
    S = built(gpu_tables, g)
    selfv, slot = S.pair_terms(btam.FP64)
    us, k, entry = p["hot_cell_us"], p["hot_cell_k"], p["hot_cell_entry"]
    gold = np.column_stack([p["hot_cell_g4"], p["hot_cell_gx"]])
    dev = device_rows(p, "hot_cell", selfv, slot)
    raw_dev = np.zeros((len(us), 5))
    raw_ref = np.zeros((len(us), 5))
    np.add.at(raw_dev, k, dev)
    np.add.at(raw_ref, k, gold)
    assert close(raw_dev, raw_ref, 1e-10)
    # weights beta_i / beta_u: i = u for the self entry, else the entry's owner
    n = len(g["x"])
    beta, owner, idx = g["beta"], g["owner"], g["idx"]
    i_of = np.where(entry < 0, us[k], owner[idx[np.maximum(entry, 0)]])
    w = beta[i_of] / beta[us[k]]
    weighted = np.zeros((len(us), 5))
    np.add.at(weighted, k, w[:, None] * dev)
    out = S.evaluate(btam.FP64)
    x, sig, b = g["x"][us], g["sigma"][us], beta[us]
    act = x >= 5e-4
    Rq = out["Rq"][us]
    Rs = out["Rs"][us] + np.where(act, 3.0 / (b * sig), 0.0)
    assert close(weighted[:, :3], Rq, 1e-10) and close(weighted[:, 3], Rs, 1e-10)
    # and the assembled residuals themselves against the reference's
    rs = p["hot_cell_res_sites"]
    assert close(out["Rq"][rs], p["hot_cell_Rq"], 1e-10)
    assert close(out["Rs"][rs], p["hot_cell_Rs"], 1e-10)
    assert close(out["Rx"][rs], p["hot_cell_Rx"], 1e-10)
    assert n == len(g["beta"]) and np.ptp(beta) > 0.0
