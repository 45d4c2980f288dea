"""The occupancy gradients alone (btam_mf_eval_x), the master equation's
chemical potentials, against the full evaluation.

R_x is evaluate_DV0_i_Dxi_u_adp_MgHx (MgHx-mf-V-bulk.cpp:2102-2325)
assembled over i in {u} U N(u).  The x-only form evaluates the same terms
from the same expressions (the values at the 13 triplet geometries without
their derivatives, the pair rule's four occupancy-free sums).  Pass 1 is
unchanged, so rho-bar, V0 and S0 equal the full evaluation's bit for bit;
R_x agrees to the last bits only, because the compiler may fuse a multiply
and an add of the shared expressions differently once the derivative terms
are gone: FP64 within 1e-13 of max(1, |R_x|), FP32C (whose sums are
compensated in FP32) within 1e-6.  The master equation keeps the pair-rule
sums between its steps (positions and widths do not move): n steps in one
call must equal n calls of one step, bit for bit, and each step must equal
the oracle's update from the device's chemical potentials (integer quanta),
which agree with the full evaluation's R_x to the same tolerance."""
import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu
RX_TOL = {btam.FP64: 1e-13, btam.FP32C: 1e-6}

# undirected shapes: plain, persistent (8, 2, 16) with (256, 2), and the
# shared-memory pass-2 shape
SHAPES = [(16, 16), (16 | 8 | 3, 16 | 8 | 3), (16 | 2, 16 | 4)]


def with_empty_sites(s, every=7):
    """Every `every`-th H site emptied (x below min_occupancy, some 0)."""
    s = dict(s)
    x = s["x"].copy()
    h = np.flatnonzero(s["species"] == 1)[::every]
    x[h] = np.where(np.arange(len(h)) % 2 == 0, 1e-4, 0.0)
    s["x"] = x
    return s


def mgh_cell(seed):
    return with_empty_sites(lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.6,
                                              x_range=(0.0, 0.6), sigma_range=(0.08, 0.15),
                                              jitter=0.02, seed=seed))


def systems():
    yield "mgh_cell", mgh_cell(5)
    yield "sphere", with_empty_sites(
        lattice.cluster("sphere", 9.0, x_fn=lambda g, rr, n: g.uniform(0.0, 0.5, n),
                        h_fraction=0.5, seed=11))


@pytest.mark.parametrize("prec", [btam.FP64, btam.FP32C])
def test_x_only_equals_full_evaluation(gpu_tables, prec):
    for name, s in systems():
        S = btam.System(gpu_tables, s)
        S.build_neighbors()
        # some H sites must be empty (x < min_occupancy) for the test to
        # cover pairs that the x-only sums include and the consumers skip
        assert np.any((s["species"] == 1) & (s["x"] < 5e-4)), name
        for v1, v2 in SHAPES:
            S.set_variants(prec, v1, v2)
            full = S.evaluate(prec)
            xo = S.evaluate_x(prec)
            for k in ("rho", "V0", "S0"):
                assert np.array_equal(xo[k], full[k]), (name, v1, v2, k)
            err = np.abs(xo["Rx"] - full["Rx"]).max()
            print(name, prec, v1, v2, "Rx max diff", err)
            assert err <= RX_TOL[prec] * max(1.0, np.abs(full["Rx"]).max()), (name, v1, v2)
            assert not np.any(xo["Rq"]) and not np.any(xo["Rs"])
            # a full evaluation afterwards is unaffected by the x-only one
            again = S.evaluate(prec)
            for k in ("Rq", "Rs", "Rx", "V0"):
                assert np.array_equal(again[k], full[k]), (name, v1, v2, k)


@pytest.mark.parametrize("prec", [btam.FP64, btam.FP32C])
def test_master_equation_keeps_pair_sums_between_steps(gpu_tables, prec):
    s = mgh_cell(7)
    prm = dict(dt=1e-3, Df=0.045, dr=3.2, min_dx=1e-8, max_x=0.9)
    A = btam.System(gpu_tables, s)
    B = btam.System(gpu_tables, s)
    for S in (A, B):
        S.build_neighbors()
        S.set_variants(prec, 16 | 8 | 3, 16 | 8 | 3)
        S.dmd_setup()
    tA = A.dmd_step(6, prec, **prm)
    for _ in range(6):
        tB = B.dmd_step(1, prec, **prm)
    xa, Xa, mua = A.dmd_occupancy()
    xb, Xb, mub = B.dmd_occupancy()
    assert tA == tB
    assert np.array_equal(Xa, Xb) and np.array_equal(mua, mub)


def test_master_equation_undirected_matches_oracle(gpu_tables, oracle):
    """Steps on the undirected kernels (x-only chemical potentials, kept
    pair sums): each update is the oracle's from the device's chemical
    potentials, total hydrogen exact, and the potentials are the full
    evaluation's R_x of the same state."""
    import pyoracle
    s = mgh_cell(5)
    n = len(s["x"])
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    S.set_variants(btam.FP64, 16 | 8 | 3, 16 | 8 | 3)
    S.dmd_setup()
    _, X0, _ = S.dmd_occupancy()
    total0 = int(X0[s["species"] == 1].sum())
    prm = dict(dt=1e-3, Df=0.045, dr=3.2, min_dx=1e-8, max_x=0.9)
    for step in range(3):
        xb, Xb, _ = S.dmd_occupancy()
        ref = S.evaluate(btam.FP64)  # the full evaluation at this state
        total = S.dmd_step(1, btam.FP64, **prm)
        assert total == total0
        x1, X1, mu = S.dmd_occupancy()
        h = (s["species"] == 1) & (xb >= 5e-4) & (xb < 0.9999)
        assert h.sum() > 10
        want = ref["Rx"][h] + s["gamma"][h] / s["beta"][h]
        assert np.abs(mu[h] - want).max() <= RX_TOL[btam.FP64] * max(1.0, np.abs(want).max())
        qg, og, _ = S.ghosts()
        owner = np.concatenate([np.arange(n), og]).astype(np.int32)
        code_all = (s["species"][owner] == 1).astype(np.int32)
        moffs, midx = S.neighbors()
        doffs, didx = S.dmd_graph()
        Xo = pyoracle.dmd_update(oracle, Xb, code_all, owner, xb[owner], s["beta"], mu, moffs,
                                 midx, doffs, didx, [prm[k] for k in ("dt", "Df", "dr",
                                                                      "min_dx", "max_x")])
        assert np.array_equal(Xo, X1), step
