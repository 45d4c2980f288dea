"""The product's per-pair arithmetic (bt-am_b200/csrc/adp_core.cuh, compiled
for the host by tests/hostmodel) against the reference's values.

This checks the moment decomposition of the triplet sums on the CPU, with
the same code the CUDA kernels run; the GPU tests then check the kernels'
work distribution.  Tolerances: FP64 1e-10 relative on per-site energies and
1e-10 (relative to the largest component) on residuals; FP32 form <= 1e-6
relative total energy and <= 1e-5 eV/A (or eV, 1/... per component) residual."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["sphere", "x5cube", "ortho_mgh", "config1"]


def load(name):
    return dict(np.load(os.path.join(GOLD, f"{name}.npz")))


def full_of(g):
    owner = g["owner"]
    full = dict(q=np.ascontiguousarray(g["q_all"]),
                sigma=np.ascontiguousarray(g["sigma"][owner]),
                x=np.ascontiguousarray(g["x"][owner]),
                species=np.ascontiguousarray(g["species"][owner]),
                beta=np.ascontiguousarray(g["beta"][owner]),
                gamma=np.ascontiguousarray(g["gamma"][owner]))
    return full


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("sym", [False, True], ids=["directed", "undirected"])
@pytest.mark.parametrize("name", NAMES)
def test_fp64_decomposition_matches_reference(hostmodel, name, sym):
    """Directed pass 2 (each site over its neighbours) and undirected pass 2
    (each pair once, both directions from its shared geometries) against the
    reference's values."""
    g = load(name)
    n = len(g["x"])
    out = hostmodel.evaluate(full_of(g), n, g["owner"], g["offs"], g["idx"], sym=sym)
    assert rel(out["rho"], g["rho"]) < 1e-12
    assert np.max(np.abs(out["V0"] - g["V0"]) / np.maximum(np.abs(g["V0"]), 1e-3)) < 1e-10
    assert rel(out["S0"], g["S0"]) < 1e-12
    us = g["res_sites"]
    scale = max(1.0, np.abs(g["Rq"]).max())
    assert np.max(np.abs(out["Rq"][us] - g["Rq"])) < 1e-10 * scale
    assert np.max(np.abs(out["Rs"][us] - g["Rs"])) < 1e-10 * max(1.0, np.abs(g["Rs"]).max())
    assert np.max(np.abs(out["Rx"][us] - g["Rx"])) < 1e-10 * max(1.0, np.abs(g["Rx"]).max())


@pytest.mark.parametrize("sym", [False, True], ids=["directed", "undirected"])
@pytest.mark.parametrize("name", NAMES)
def test_fp32_form_within_tolerance(hostmodel, name, sym):
    g = load(name)
    n = len(g["x"])
    out = hostmodel.evaluate(full_of(g), n, g["owner"], g["offs"], g["idx"], fp32=True, sym=sym)
    E, E0 = out["V0"].sum(), g["V0"].sum()
    assert abs(E - E0) <= 1e-6 * abs(E0)
    us = g["res_sites"]
    assert np.max(np.abs(out["Rq"][us] - g["Rq"])) <= 1e-5
    assert np.max(np.abs(out["Rs"][us] - g["Rs"])) <= 1e-5
    assert np.max(np.abs(out["Rx"][us] - g["Rx"])) <= 1e-5 * max(1.0, np.abs(g["Rx"]).max())


@pytest.mark.parametrize("name", NAMES)
def test_undirected_equals_directed(hostmodel, name):
    """Both pass-2 forms in FP64 agree to rounding on every site."""
    g = load(name)
    n = len(g["x"])
    a = hostmodel.evaluate(full_of(g), n, g["owner"], g["offs"], g["idx"])
    b = hostmodel.evaluate(full_of(g), n, g["owner"], g["offs"], g["idx"], sym=True)
    for k in ("Rq", "Rs", "Rx"):
        assert np.max(np.abs(a[k] - b[k])) <= 1e-12 * max(1.0, np.abs(a[k]).max()), k


def test_inactive_hydrogen_and_translation_invariance(hostmodel, oracle):
    """Empty H sites (x < 5e-4) contribute nothing and get zero residuals;
    a periodic system's q-residuals sum to zero (translation invariance)."""
    import pyoracle
    from btam import lattice
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.5, x_range=(0.0, 0.02),
                          jitter=0.03, seed=21)
    full, n, owner, image = pyoracle.expand(s, oracle)
    offs, idx = oracle.neighbors(full["q"])
    out = hostmodel.evaluate(full, n, owner, offs, idx)
    empty = s["x"] < 5e-4
    assert empty.any()
    assert np.all(out["V0"][empty] == 0.0) and np.all(out["Rq"][empty] == 0.0)
    assert np.all(out["Rx"][empty] == 0.0)
    assert np.abs(out["Rq"].sum(axis=0)).max() < 1e-10 * np.abs(out["Rq"]).max() * n
