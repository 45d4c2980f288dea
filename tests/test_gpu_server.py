"""Job server: results of every job alone and in a concurrent mix.

Tolerance: none.  The server merges the evaluations of the running jobs into
shared batched launches (continuous batching); every kernel is
deterministic, a job's rows never mix with another's and the kernel shapes
are fixed, so a job's final state, residual norm, objective and hydrogen
total must be bitwise the same whether it ran alone or in a mix."""
import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu


def job_mix():
    cell = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.4, x_range=(0.2, 0.5),
                             sigma_range=(0.08, 0.15), jitter=0.02, seed=21)
    hexa = lattice.supercell(5, 5, 4, ortho=False, h_fraction=0.5, x_range=(0.0, 0.4),
                             sigma_range=(0.08, 0.15), jitter=0.02, seed=22)
    sph = lattice.sphere(10.0, T=450.0, h_fraction=0.3, seed=23)
    sph2 = lattice.sphere(13.0, T=350.0, h_fraction=0.45, seed=24)
    return [
        (cell, dict(kind=btam.JOB_RELAX, mode=btam.RELAX_FP32C, tol=1e-5, max_iter=120)),
        (hexa, dict(kind=btam.JOB_DMD, precision=btam.FP32C, nsteps=20)),
        (sph, dict(kind=btam.JOB_RELAX, mode=btam.RELAX_MIXED, tol=1e-7, max_iter=200)),
        (sph2, dict(kind=btam.JOB_DMD, precision=btam.FP64, nsteps=10)),
        (hexa, dict(kind=btam.JOB_EVAL, precision=btam.FP32C)),
        (sph2, dict(kind=btam.JOB_EVAL, precision=btam.FP64)),
        (cell, dict(kind=btam.JOB_STRETCH, tol=1e-12, max_iter=20)),
        (sph, dict(kind=btam.JOB_RELAX, mode=btam.RELAX_NEWTON, tol=1e-7, max_iter=40)),
        (cell, dict(kind=btam.JOB_RELAX, mode=btam.RELAX_NGMRES, tol=1e-7, max_iter=150)),
    ]


KEYS = ("status", "norm", "objective", "iterations", "evaluations", "converged", "h_quanta")


def same(a, b):
    for k in KEYS:
        assert a[k] == b[k], k
    for k in ("q", "sigma", "x"):
        assert np.array_equal(a[k], b[k]), k


def test_server_results_alone_equal_in_mix(gpu_tables):
    jobs = job_mix()
    alone = []
    srv = btam.Server(gpu_tables, workers=1)
    for s, kw in jobs:
        alone.append(srv.wait(srv.submit(s, **kw)))
    srv.close()
    srv = btam.Server(gpu_tables, workers=6)
    ids = [srv.submit(s, **kw) for s, kw in jobs for _ in range(2)]
    mixed = [srv.wait(i) for i in ids]
    st = srv.stats()
    bs = srv.batch_stats()
    srv.close()
    assert st["completed"] >= len(ids) and st["failed"] == 0
    # evaluations were shared: rounds served several jobs at once
    assert bs["evaluations"] > bs["rounds"] > 0 and bs["rebuilds"] > 0
    for k, r in enumerate(mixed):
        same(alone[k // 2], r)
    # the jobs did overlap: some job started before another had ended
    spans = sorted((r["t_start"], r["t_end"]) for r in mixed)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    # an evaluation job equals the direct evaluation of the system
    S = btam.System(gpu_tables, jobs[4][0])
    S.build_neighbors()
    S.set_variants(btam.FP32C, 16 | 8 | 3, 16 | 8 | 2)  # the server's FP32C launch variants
    tot = S.evaluate(btam.FP32C)["totals"]
    assert alone[4]["objective"] == tot[0] and alone[4]["norm"] == tot[2]


def test_server_admission_by_memory(gpu_tables):
    """A budget that holds about two of these jobs at once: all still finish,
    never more than the budget is admitted, and a job larger than the whole
    budget is refused at submission."""
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.4, x_range=(0.0, 0.3), seed=31)
    need = btam.estimate_bytes(s)
    srv = btam.Server(gpu_tables, workers=8, budget_bytes=int(2.5 * need))
    ids = [srv.submit(s, kind=btam.JOB_DMD, precision=btam.FP32C, nsteps=5) for _ in range(6)]
    peak = 0
    out = []
    for i in ids:
        peak = max(peak, srv.stats()["bytes_in_use"])
        out.append(srv.wait(i))
    assert peak <= int(2.5 * need)
    for r in out[1:]:
        assert r["h_quanta"] == out[0]["h_quanta"] and np.array_equal(r["x"], out[0]["x"])
    big = lattice.supercell(12, 8, 8, ortho=True, h_fraction=0.4, seed=32)
    assert btam.estimate_bytes(big) > 2.5 * need
    with pytest.raises(btam.BtamError) as e:
        srv.submit(big, kind=btam.JOB_EVAL)
    assert e.value.code == 15
    srv.close()


def test_stretch_newton_and_ngmres_jobs_equal_direct_calls(gpu_tables):
    """A bulk stretch job, a Newton relaxation job and an N-GMRES(3)
    relaxation job give the final state, residual and counts of the same
    calls made directly on a system."""
    jobs = job_mix()
    cell, kw_s = jobs[6]
    sph, kw_n = jobs[7]
    cell_g, kw_g = jobs[8]
    srv = btam.Server(gpu_tables, workers=2)
    rs = srv.wait(srv.submit(cell, **kw_s))
    rn = srv.wait(srv.submit(sph, **kw_n))
    rg = srv.wait(srv.submit(cell_g, **kw_g))
    srv.close()
    G = btam.System(gpu_tables, cell_g)
    G.build_neighbors()
    G.set_variants(btam.FP64, 16 | 8 | 3, 16 | 8 | 0)
    info = G.relax(mode=btam.RELAX_NGMRES, tol=1e-7, max_iter=150, m=3)
    qg, sg, _ = G.get_state()
    assert rg["status"] == 0 and rg["converged"] == info["status"], (rg, info)
    assert rg["iterations"] == info["iterations"] == 150 or info["status"] == 1
    assert rg["norm"] == info["norm"] and rg["evaluations"] == info["evaluations"]
    assert np.array_equal(rg["q"], qg) and np.array_equal(rg["sigma"], sg)
    S = btam.System(gpu_tables, cell)
    S.build_neighbors()
    F, info = S.relax_stretch(atol=1e-12, rtol=1e-10, max_iter=20)
    q, _, _ = S.get_state()
    assert rs["status"] == 0 and rs["converged"] == 1 and info["status"] == 1
    assert np.array_equal(rs["q"], q) and rs["objective"] == F[0] * F[1] * F[2]
    N = btam.System(gpu_tables, sph)
    N.build_neighbors()
    N.set_variants(btam.FP64, 16 | 8 | 3, 16 | 8 | 0)
    info = N.relax_newton(tol=1e-7, max_newton=40, max_cg=300)
    qn, sn, _ = N.get_state()
    assert rn["status"] == 0 and rn["converged"] == info["status"]
    assert rn["norm"] == info["norm"] and rn["evaluations"] == info["evaluations"]
    assert np.array_equal(rn["q"], qn) and np.array_equal(rn["sigma"], sn)
