"""The consumers of the evaluation on the GPU: (q, sigma) relaxation and the
hydrogen master equation, against their oracle definitions.

Tolerances: relaxation to the requested residual norm, checked again with
the literal oracle residuals of the relaxed state (<= 10 x tol); the
master-equation update bit-exact in integer quanta given the same chemical
potentials; total hydrogen conserved exactly (integer equality)."""
import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu


def small_mgh(seed=5, h=0.3, xr=(0.0, 0.4)):
    return lattice.supercell(4, 3, 3, ortho=True, h_fraction=h, x_range=xr,
                             sigma_range=(0.08, 0.15), jitter=0.02, seed=seed)


@pytest.mark.parametrize("mode", [0, 1, 4])
def test_relaxation_reaches_tolerance(gpu_tables, oracle, mode):
    """Well-occupied Mg-H cell: every site relaxes and the projected
    residual reaches 1e-8 (mode 4: N-GMRES(3) with the critical-point line
    search, the reference's SNES options); the literal oracle agrees the
    state is stationary."""
    import pyoracle
    s = small_mgh(xr=(0.3, 0.6))
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    info = S.relax(mode=mode, tol=1e-8, max_iter=2000 if mode == 4 else 600,
                   m=3 if mode == 4 else 8)
    assert info["status"] == 1 and info["norm"] <= 1e-8, info
    q, sigma, x = S.get_state()
    assert np.all(sigma < 0.4)  # no bound active here, so the full residual vanishes
    out = S.evaluate(btam.FP64)
    assert np.sqrt(out["totals"][2]) <= 1e-8
    # literal residuals on the same (fixed) images and neighbour lists
    r = dict(s, q=q, sigma=sigma, x=x)
    qg, og, ig = S.ghosts()
    offs, idx = S.neighbors()
    sites = np.array([0, 7, 40, 150, 200], np.int32)
    lit = pyoracle.residuals_on_topology(oracle, r, qg, og, ig, offs, idx, sites)
    assert np.abs(lit["Rq"]).max() <= 1e-7 and np.abs(lit["Rs"]).max() <= 1e-7


def test_relaxation_dilute_hydrogen_config1(gpu_tables):
    """Config 1 (x ~ U[0, 0.1]): sites below x_min stay fixed, sigma bounds
    hold; the projected residual falls by orders of magnitude."""
    s = lattice.config1()
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    r0 = np.sqrt(S.evaluate(btam.FP64)["totals"][2])
    info = S.relax(mode=1, tol=1e-8, max_iter=800)
    q, sigma, x = S.get_state()
    assert np.all((sigma >= 0.001 - 1e-15) & (sigma <= 0.4 + 1e-12))
    fixed = s["x"] < 0.01
    assert np.array_equal(q[fixed], s["q"][fixed]) and np.array_equal(sigma[fixed],
                                                                        s["sigma"][fixed])
    assert info["norm"] < 1e-4 * r0, info


def test_newton_relaxation_stationary_by_oracle(gpu_tables, oracle):
    """The Newton option on the well-occupied cell: converged, and the
    literal oracle residuals of the relaxed state vanish."""
    import pyoracle
    s = small_mgh(xr=(0.3, 0.6))
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    info = S.relax_newton(tol=1e-8, max_newton=100, max_cg=300)
    assert info["status"] == 1 and info["norm"] <= 1e-8, info
    q, sigma, x = S.get_state()
    r = dict(s, q=q, sigma=sigma, x=x)
    qg, og, ig = S.ghosts()
    offs, idx = S.neighbors()
    sites = np.array([0, 7, 40, 150, 200], np.int32)
    lit = pyoracle.residuals_on_topology(oracle, r, qg, og, ig, offs, idx, sites)
    assert np.abs(lit["Rq"]).max() <= 1e-7 and np.abs(lit["Rs"]).max() <= 1e-7


def test_newton_relaxation_config1_stationary(gpu_tables, oracle):
    """Config 1 (dilute H, sigma bounds active): the Newton option and L-BFGS
    both reach 1e-8, and the literal oracle's residuals vanish at the Newton
    state on sampled relaxed sites; held sites stay fixed.  The dilute
    landscape has minima that differ by about 2e-7 relative in F (which one a
    solver reaches changes with the last bits of the evaluations), so the
    two objectives are compared to 1e-6 relative only."""
    import pyoracle
    s = lattice.config1()
    A = btam.System(gpu_tables, s)
    A.build_neighbors()
    ia = A.relax(mode=0, tol=1e-8, max_iter=2000)
    B = btam.System(gpu_tables, s)
    B.build_neighbors()
    ib = B.relax_newton(tol=1e-8, max_newton=100, max_cg=300)
    assert ia["status"] == 1 and ib["status"] == 1, (ia, ib)
    assert abs(ia["objective"] - ib["objective"]) <= 1e-6 * abs(ia["objective"])
    qb, sb, xb = B.get_state()
    fixed = s["x"] < 0.01
    r = dict(s, q=qb, sigma=sb, x=xb)
    qg, og, ig = B.ghosts()
    offs, idx = B.neighbors()
    relaxed = np.flatnonzero(~fixed)
    sites = relaxed[:: max(1, len(relaxed) // 8)].astype(np.int32)
    lit = pyoracle.residuals_on_topology(oracle, r, qg, og, ig, offs, idx, sites)
    assert np.abs(lit["Rq"]).max() <= 1e-7
    inside = (sb[sites] > 0.001 * (1 + 1e-9)) & (sb[sites] < 0.4 * (1 - 1e-9))
    assert np.abs(lit["Rs"][inside]).max(initial=0.0) <= 1e-7
    assert np.array_equal(qb[fixed], s["q"][fixed])
    assert np.all((sb >= 0.001 - 1e-15) & (sb <= 0.4 + 1e-12))


def test_ngmres_relaxation_config1_stationary(gpu_tables, oracle):
    """Config 1 (dilute H, sigma bounds active): N-GMRES(3) with the
    critical-point line search reaches 1e-8 with three evaluations per
    iteration; the literal oracle's residuals of the relaxed state vanish on
    sampled relaxed sites (R_sigma where sigma is inside its bounds); held
    sites stay fixed.  N-GMRES solves g = 0, so on this landscape it may stop
    at another stationary point than the descent methods (its objective is
    compared with theirs only to 1e-5 relative)."""
    import pyoracle
    s = lattice.config1()
    A = btam.System(gpu_tables, s)
    A.build_neighbors()
    ia = A.relax(mode=btam.RELAX_NGMRES, tol=1e-8, max_iter=20000, m=3)
    assert ia["status"] == 1 and ia["norm"] <= 1e-8, ia
    assert ia["evaluations"] <= 1 + 3 * ia["iterations"], ia
    B = btam.System(gpu_tables, s)
    B.build_neighbors()
    ib = B.relax_newton(tol=1e-8, max_newton=100, max_cg=300)
    assert abs(ia["objective"] - ib["objective"]) <= 1e-5 * abs(ib["objective"]), (ia, ib)
    q, sigma, x = A.get_state()
    fixed = s["x"] < 0.01
    assert np.array_equal(q[fixed], s["q"][fixed])
    assert np.array_equal(sigma[fixed], s["sigma"][fixed])
    assert np.all((sigma >= 0.001 - 1e-15) & (sigma <= 0.4 + 1e-12))
    r = dict(s, q=q, sigma=sigma, x=x)
    qg, og, ig = A.ghosts()
    offs, idx = A.neighbors()
    relaxed = np.flatnonzero(~fixed)
    h = relaxed[s["species"][relaxed] == 1]
    sites = np.concatenate([relaxed[:: max(1, len(relaxed) // 6)], h[:6]]).astype(np.int32)
    lit = pyoracle.residuals_on_topology(oracle, r, qg, og, ig, offs, idx, sites)
    assert np.abs(lit["Rq"]).max() <= 1e-7, np.abs(lit["Rq"]).max()
    inside = (sigma[sites] > 0.001 * (1 + 1e-9)) & (sigma[sites] < 0.4 * (1 - 1e-9))
    assert np.abs(lit["Rs"][inside]).max(initial=0.0) <= 1e-7


def test_diffusive_graph_bit_exact(gpu_tables):
    import pyoracle
    s = small_mgh(h=0.6)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    S.dmd_setup()
    offs, idx = S.dmd_graph()
    qg, og, _ = S.ghosts()
    n = len(s["x"])
    q_all = np.concatenate([s["q"], qg])
    sp_all = np.concatenate([s["species"], s["species"][og]])
    o2, i2 = pyoracle.diffusive_graph(q_all, sp_all, n)
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)


def test_master_equation_matches_oracle_and_conserves(gpu_tables, oracle):
    import pyoracle
    s = small_mgh(h=0.6, xr=(0.0, 0.6))
    n = len(s["x"])
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    S.dmd_setup()
    x0, X0, _ = S.dmd_occupancy()
    total0 = int(X0[s["species"] == 1].sum())
    prm = dict(dt=1e-3, Df=0.045, dr=3.2, min_dx=1e-8, max_x=0.9)
    for step in range(3):
        xb, Xb, _ = S.dmd_occupancy()
        total = S.dmd_step(1, btam.FP64, **prm)
        assert total == total0  # exact conservation
        x1, X1, mu = S.dmd_occupancy()
        # the oracle's update from the same chemical potentials and state
        qg, og, _ = S.ghosts()
        owner = np.concatenate([np.arange(n), og]).astype(np.int32)
        code_all = (s["species"][owner] == 1).astype(np.int32)
        x_all = xb[owner]
        moffs, midx = S.neighbors()
        doffs, didx = S.dmd_graph()
        Xo = pyoracle.dmd_update(oracle, Xb, code_all, owner, x_all, s["beta"], mu, moffs, midx,
                                 doffs, didx, [prm[k] for k in ("dt", "Df", "dr", "min_dx",
                                                                "max_x")])
        assert np.array_equal(Xo, X1), step
        assert np.any(X1 != Xb)


def dmd_context(S, s, xb):
    """The arguments the oracle's master-equation functions take, from a
    device system and the occupancies xb of its real sites."""
    n = len(s["x"])
    qg, og, _ = S.ghosts()
    owner = np.concatenate([np.arange(n), og]).astype(np.int32)
    code_all = (s["species"][owner] == 1).astype(np.int32)
    moffs, midx = S.neighbors()
    doffs, didx = S.dmd_graph()
    return dict(code_all=code_all, owner=owner, x_all=xb[owner], beta=s["beta"], moffs=moffs,
                midx=midx, doffs=doffs, didx=didx)


def test_master_equation_step_control_matches_oracle(gpu_tables, oracle):
    """A controlled step: the device's decision equals the oracle's at the
    same chemical potentials, the step equals m plain steps of dt / m (each
    the oracle's update of its state), the clipped moves are the oracle's,
    and total hydrogen is exact."""
    import pyoracle
    s = small_mgh(h=0.6, xr=(0.0, 0.6))
    prm = dict(dt=2e-3, Df=0.045, dr=3.2, min_dx=1e-8, max_x=0.9)
    plist = [prm[k] for k in ("dt", "Df", "dr", "min_dx", "max_x")]
    A, B = (btam.System(gpu_tables, s) for _ in range(2))
    for S in (A, B):
        S.build_neighbors()
        S.dmd_setup()
    # the chemical potentials at the start (a step of dt = 0 moves nothing)
    total0 = B.dmd_step(1, btam.FP64, **dict(prm, dt=0.0))
    x0, X0, mu0 = B.dmd_occupancy()
    ctx = dmd_context(B, s, x0)
    r = pyoracle.dmd_control(oracle, X0, mu=mu0, params=plist, max_dx=1.0, **ctx)
    # a site-change bound that needs several sub-steps
    max_dx = r[1] / 3.5
    r = pyoracle.dmd_control(oracle, X0, mu=mu0, params=plist, max_dx=max_dx, **ctx)
    m = int(max(1, np.ceil(max(r))))
    assert m >= 4
    total, st = A.dmd_step_ctl(1, btam.FP64, max_dx=max_dx, **prm)
    assert st["substeps"] == m and st["subdivided"] == 1 and total == total0
    assert abs(st["worst_ratio"] - max(r)) <= 1e-12 * max(r)
    clips = 0
    for j in range(m):
        xb, Xb, _ = B.dmd_occupancy()
        B.dmd_step(1, btam.FP64, **dict(prm, dt=prm["dt"] / m))
        _, X1, mu = B.dmd_occupancy()
        Xo, c = pyoracle.dmd_update(oracle, Xb, mu=mu, params=[prm["dt"] / m] + plist[1:],
                                    count_clips=True, **dmd_context(B, s, xb))
        assert np.array_equal(Xo, X1), j
        clips += c
    _, XA, _ = A.dmd_occupancy()
    assert np.array_equal(XA, X1)
    assert st["clipped"] == clips and A.dmd_clip_count() == clips


def test_master_equation_clipping_is_counted(gpu_tables, oracle):
    """A step long enough that moves are cut to their room: the plain step
    counts the cut moves as the oracle does; the controlled step divides it
    until none is cut, and conserves hydrogen exactly."""
    import pyoracle
    s = small_mgh(h=0.8, xr=(0.0, 0.6), seed=13)
    prm = dict(dt=0.5, Df=0.045, dr=3.2, min_dx=1e-8, max_x=0.9)
    plist = [prm[k] for k in ("dt", "Df", "dr", "min_dx", "max_x")]
    A, B = (btam.System(gpu_tables, s) for _ in range(2))
    for S in (A, B):
        S.build_neighbors()
        S.dmd_setup()
    xb, Xb, _ = B.dmd_occupancy()
    total0 = B.dmd_step(1, btam.FP64, **prm)
    _, X1, mu = B.dmd_occupancy()
    Xo, c = pyoracle.dmd_update(oracle, Xb, mu=mu, params=plist, count_clips=True,
                                **dmd_context(B, s, xb))
    assert np.array_equal(Xo, X1) and c > 0 and B.dmd_clip_count() == c
    total, st = A.dmd_step_ctl(1, btam.FP64, max_dx=1.0, max_sub=4096, **prm)
    assert total == total0 and st["substeps"] > 1 and st["worst_ratio"] > 1.0
    assert A.dmd_clip_count() == st["clipped"]


def test_dmd_run_relaxes_between_steps(gpu_tables):
    """btam_dmd_run equals its parts run by hand (controlled steps, then a
    relaxation every k steps), bit for bit, and conserves hydrogen."""
    s = small_mgh(h=0.6, xr=(0.05, 0.6), seed=17)
    A, B = (btam.System(gpu_tables, s) for _ in range(2))
    for S in (A, B):
        S.build_neighbors()
        S.dmd_setup()
    total0 = B.dmd_step(0, btam.FP64)
    total, st = A.dmd_run(6, btam.FP64, relax_every=3, relax_tol=1e-6, relax_max_iter=100,
                          dt=1e-3)
    assert total == total0 and st["relaxations"] == 2 and st["relax_evaluations"] > 0
    for _ in range(2):
        B.dmd_step_ctl(3, btam.FP64, dt=1e-3)
        B.relax(mode=0, tol=1e-6, max_iter=100, m=8)
    for a, b in zip(A.get_state(), B.get_state()):
        assert np.array_equal(a, b)
    assert np.array_equal(A.dmd_occupancy()[1], B.dmd_occupancy()[1])


def test_master_equation_long_run_conserves_and_bounds(gpu_tables):
    s = small_mgh(h=0.8, xr=(0.0, 0.5), seed=9)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    S.dmd_setup()
    _, X0, _ = S.dmd_occupancy()
    total0 = int(X0[s["species"] == 1].sum())
    total = S.dmd_step(200, btam.FP32C, dt=1e-3)
    assert total == total0
    x, X, mu = S.dmd_occupancy()
    h = s["species"] == 1
    assert np.all(X[h] >= 0) and np.all(x[h] <= 0.9 + 1e-12)
    assert np.all(np.isfinite(mu))
    assert np.array_equal(x[h], X[h] * 2.0 ** -50)


def test_master_equation_nanowire_conserves(gpu_tables):
    """The precision workload's system (hcp Mg nanowire, radius 30 A, 20
    cells, periodic along the axis, H x ~ U[0, 0.5] beyond 20 A): FP32C
    residuals, FP64 occupancy updates; total hydrogen exact to the quantum
    and occupancies inside [0, 0.9] after 50 steps."""
    s = lattice.config3()
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    S.dmd_setup()
    total0 = S.dmd_step(0, btam.FP32C, dt=1e-3)
    total = S.dmd_step(50, btam.FP32C, dt=1e-3)
    assert total == total0
    x, X, mu = S.dmd_occupancy()
    h = s["species"] == 1
    assert np.all(X[h] >= 0) and np.all(x[h] <= 0.9 + 1e-12) and np.all(np.isfinite(mu))
    assert np.abs(x[h] - s["x"][h]).max() > 0.0  # hydrogen moved
    # the same steps with step control report what they did
    total, st = S.dmd_step_ctl(20, btam.FP32C, dt=1e-3)
    assert total == total0 and st["substeps"] >= 20
    assert st["clipped"] >= 0 and np.isfinite(st["worst_ratio"])


def test_master_equation_checkpoint_resume_bitwise(gpu_tables, tmp_path):
    """Checkpoint / resume through the reference's dump format: 20 steps,
    the device state written as a dump and read into a new system, 20 more
    steps give the same occupancy quanta, to the bit, as 40 steps in one
    run (occupancies are exact multiples of the quantum, the dump keeps
    every double exactly, and every kernel is deterministic)."""
    from btam import dump
    s = small_mgh(h=0.6, xr=(0.0, 0.5), seed=13)
    A = btam.System(gpu_tables, s)
    A.build_neighbors()
    A.dmd_setup()
    A.dmd_step(40, btam.FP32C, dt=1e-3)
    _, XA, _ = A.dmd_occupancy()
    B = btam.System(gpu_tables, s)
    B.build_neighbors()
    B.dmd_setup()
    B.dmd_step(20, btam.FP32C, dt=1e-3)
    q, sigma, x = B.get_state()
    path = str(tmp_path / "checkpoint.dump")
    dump.write_dump(path, dict(s, q=q, sigma=sigma, x=x), timestep=20)
    r = dump.read_dump(path)
    assert r["timestep"] == 20 and np.array_equal(r["x"], x)
    C = btam.System(gpu_tables, r)
    C.build_neighbors()
    C.dmd_setup()
    C.dmd_step(20, btam.FP32C, dt=1e-3)
    _, XC, _ = C.dmd_occupancy()
    assert np.array_equal(XA, XC)
