"""Batched evaluation (many systems, one graph launch per evaluation) against
each system evaluated on its own.

Tolerance: none.  With the same kernel block shapes, every per-site result
and every per-system total of the batch must equal the single-system result
bitwise, in both arithmetic forms, because each site is computed by the same
instructions in the same order and the per-system totals use the same
reduction tree."""
import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu

FIELDS = ("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals")


def mixed_systems():
    out = [lattice.sphere(8.5, T=350.0, h_fraction=0.4, seed=1),
           lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.3, x_range=(0.0, 0.4),
                             sigma_range=(0.08, 0.15), jitter=0.02, seed=2),
           lattice.sphere(11.0, T=550.0, h_fraction=0.1, seed=3),
           lattice.supercell(5, 5, 4, ortho=False, h_fraction=0.5, x_range=(0.0, 0.3),
                             sigma_range=(0.08, 0.15), jitter=0.02, seed=4),
           lattice.sphere(9.0, T=420.0, h_fraction=0.0, seed=5)]
    return out


def built(tables, dicts):
    systems = []
    for d in dicts:
        S = btam.System(tables, d)
        S.build_neighbors()
        systems.append(S)
    return systems


def assert_same(a, b, what):
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), (what, f, np.abs(a[f] - b[f]).max())


@pytest.mark.parametrize("und", [0, 16], ids=["directed", "undirected"])
@pytest.mark.parametrize("prec", [btam.FP64, btam.FP32C])
def test_batch_equals_single_systems_bitwise(gpu_tables, prec, und):
    systems = built(gpu_tables, mixed_systems())
    for S in systems:
        S.set_variants(prec, und, und)  # shape 0, full grid
    B = btam.Batch(systems)
    B.set_variants(prec, und | 8, und | 8)  # shape 0, persistent grid
    info = B.info()
    assert info["n_sys"] == len(systems)
    assert info["n_real"] == sum(S.n for S in systems)
    B.evaluate(prec)
    tot = B.totals()
    for k, S in enumerate(systems):
        single = S.evaluate(prec)
        assert_same(B.results(k), single, k)
        assert np.array_equal(tot[k], single["totals"])


def test_batch_state_update_and_autotune(gpu_tables):
    dicts = mixed_systems()
    systems = built(gpu_tables, dicts)
    B = btam.Batch(systems)
    B.evaluate(btam.FP32C)
    before = [B.results(k) for k in range(len(systems))]
    # new widths and occupancies of the periodic system 1 (image refresh) and
    # new positions of the sphere 0; neighbour lists stay as built
    rng = np.random.default_rng(11)
    d = dicts[1]
    sigma = d["sigma"] * rng.uniform(0.97, 1.03, d["sigma"].shape)
    x = np.where(d["species"] == 1, d["x"] * rng.uniform(0.9, 1.1, d["x"].shape), d["x"])
    B.set_state(1, sigma=sigma, x=x)
    d0 = dicts[0]
    B.set_state(0, q=d0["q"] + rng.normal(0.0, 0.003, d0["q"].shape))
    v1, v2 = B.autotune(btam.FP32C)
    assert v1 >= 0 and v2 >= 0
    B.evaluate(btam.FP32C)
    for k, S in enumerate(systems):
        S.set_variants(btam.FP32C, v1 & ~8, v2 & ~8)  # same kernels as the batch, full grid
        got = B.results(k)
        assert_same(got, S.evaluate(btam.FP32C), (k, v1, v2))
        if k > 1:  # unchanged systems: same energies (pass 1 is the same
            # arithmetic for every launch variant up to rounding)
            assert np.abs(got["V0"].sum() - before[k]["V0"].sum()) <= 1e-6 * np.abs(
                before[k]["V0"].sum())
        else:
            assert not np.array_equal(got["V0"], before[k]["V0"])


def test_batch_config4_spheres(gpu_tables):
    """The batched workload: 128 spheres of radii log-uniform on [8, 25] A,
    every system's totals equal to its own evaluation, repeated launches
    reproducible."""
    systems = built(gpu_tables, lattice.config4())
    B = btam.Batch(systems)
    v1, v2 = B.autotune(btam.FP32C)
    t1 = B.evaluate(btam.FP32C)
    t2 = B.evaluate(btam.FP32C)
    assert np.array_equal(t1, t2)
    for k in range(0, len(systems), 9):
        systems[k].set_variants(btam.FP32C, v1, v2)
        single = systems[k].evaluate(btam.FP32C)
        assert np.array_equal(t1[k], single["totals"]), k
        assert_same(B.results(k), single, k)
