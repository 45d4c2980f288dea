"""Generates the golden fixtures in tests/golden/ from the reference itself.

Values come from the reference's own arithmetic files compiled unmodified
(oracle/_ref/libbtam_ref.so, built by oracle/Makefile from the reference
tree): cubic_spline/d_cubic_spline, the Gaussian measure and degree-3 rule,
the ADP terms, evaluate_mf_rho_i / V0_i / S0_i / DV0_i_Dq_u / DV0_i_Dxi_u.
Periodic images and neighbour lists come from the restated rule
(oracle/btam_oracle.cpp), because the reference builds them with PETSc
DMSwarm, which is not available; the residual assembly is the project's
definition (include/btam.h) applied to the reference's per-pair values.

Run from the repository root, with the reference tree present:
    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --point    # point.npz only (it reads
                                                  # the system fixtures)
    python tests/golden/make_golden.py --multipole  # multipole.npz only (it
                                                    # reads the system fixtures)
    python tests/golden/make_golden.py --pairs    # pairs.npz only (it reads
                                                  # the system fixtures)
    python tests/golden/make_golden.py --termfns  # termfns.npz only
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "bt-am_b200")]
import pyoracle  # noqa: E402
from btam import dump, lattice  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
# the reference tree: $BTAM_REFERENCE, else a checkout named "reference" beside
# this repository
REF_TREE = os.environ.get("BTAM_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))


def residual_pairs(full, owner, image, offs, idx, us):
    """(u', o) argument pairs of the assembly for each u in us, as the
    restated orc_residuals forms them (images seen from the owner's frame)."""
    plan = []
    for k, u in enumerate(us):
        cen = [u] + list(idx[offs[u]:offs[u + 1]])
        for ic in cen:
            o = owner[ic]
            T = image[ic]
            uu = u
            if np.any(T != 0):
                uu = -1
                for cand in idx[offs[o]:offs[o + 1]]:
                    if owner[cand] == u and np.all(image[cand] == -T):
                        uu = cand
                        break
                if uu < 0:
                    continue
            plan.append((k, uu, o))
    return plan


def assemble(ref, full, rho, owner, image, offs, idx, us):
    plan = residual_pairs(full, owner, image, offs, idx, us)
    kk = np.array([p[0] for p in plan])
    uu = np.array([p[1] for p in plan], np.int32)
    oo = np.array([p[2] for p in plan], np.int32)
    g4, gx = ref.DV0_pairs(full, rho, offs, idx, uu, oo)
    beta, gamma, x, sig = full["beta"], full["gamma"], full["x"], full["sigma"]
    Rq = np.zeros((len(us), 3))
    Rs = np.zeros(len(us))
    Rx = np.zeros(len(us))
    for p in range(len(plan)):
        k = kk[p]
        u = us[k]
        w = beta[oo[p]] / beta[u]
        Rq[k] += w * g4[p, :3]
        Rs[k] += w * g4[p, 3]
        Rx[k] += w * gx[p]
    for k, u in enumerate(us):
        if x[u] < 5e-4:
            Rq[k] = 0.0
            Rs[k] = Rx[k] = 0.0
            continue
        Rs[k] -= 3.0 / (beta[u] * sig[u])
        if full["species"][u] == 1:
            dlogz = 3.0 / (2.0 * x[u]) + (1.0 / (1.0 - x[u]) if x[u] < 1.0 else 0.0)
            Rx[k] -= dlogz / beta[u]
            if x[u] < 0.9999:
                Rx[k] -= gamma[u] / beta[u]
        else:
            Rx[k] = 0.0
    return Rq, Rs, Rx


def system_fixture(name, s, ref, orc, residual_sample=None, seed=0):
    full, n, owner, image = pyoracle.expand(s, orc)
    offs, idx = orc.neighbors(full["q"])
    real = np.arange(n, dtype=np.int32)
    rho_real = ref.mf_rho(full, offs, idx, real)
    rho = rho_real[owner]
    V0 = ref.V0(full, rho, offs, idx, real)
    S0 = ref.S0(full, rho, offs, idx, real)
    if residual_sample is None:
        us = real
    else:
        rng = np.random.default_rng(seed)
        us = np.sort(rng.choice(n, residual_sample, replace=False)).astype(np.int32)
    Rq, Rs, Rx = assemble(ref, full, rho, owner, image, offs, idx, us)
    rho_nmf = ref.rho_nmf(full, offs, idx, real)
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(
        path, q=s["q"], sigma=s["sigma"], x=s["x"], species=s["species"], beta=s["beta"],
        gamma=s["gamma"], origin=s["origin"], cell=s["cell"], periodic=s["periodic"],
        q_all=full["q"], owner=owner, image=image, offs=offs, idx=idx, rho=rho_real, V0=V0,
        S0=S0, res_sites=us, Rq=Rq, Rs=Rs, Rx=Rx, rho_nmf=rho_nmf)
    print(f"{name}: {n} real, {len(full['x'])} sites, {len(idx)} pairs, "
          f"{len(us)} residual sites -> {os.path.getsize(path)} bytes")


# Stretch of the non-mean-field fixtures: q <- diag(F) q on every site.
PT_STRETCH = np.array([1.01, 0.99, 1.02])


def point_fixture(ref):
    """Non-mean-field forms (sigma -> 0) on the committed systems, from the
    reference's own evaluate_rho_i / evaluate_DV_i_Dq_u_adp_MgHx /
    evaluate_DV_i_dF_MgHx, on the neighbour lists stored in each fixture:
    the assembled gradient sum_{i in {u} U N(u)} dV_i/dq_u of every real
    site, the same sum of evaluate_D2V_i_Dq2_u_MgHx, dV_i/dF with q0 = q, and dV_i/dF after the stretch PT_STRETCH
    (q0 = the unstretched positions, neighbour lists kept); and the
    mean-field stretch derivative evaluate_DV0_i_dF_bulk_MgHx at q0 = q and
    after the same stretch (with the mean-field rho-bar there), and the
    assembled mean-field Hessian blocks evaluate_D2V0_i_Dmeanq2_u_MgHx."""
    out = {"stretch": PT_STRETCH}
    for name in ("sphere", "ortho_mgh", "x5cube", "config1"):
        g = np.load(os.path.join(OUT, f"{name}.npz"))
        n = len(g["x"])
        owner, image, offs, idx = g["owner"], g["image"], g["offs"], g["idx"]
        full = {"q": np.ascontiguousarray(g["q_all"]),
                "x": np.ascontiguousarray(g["x"][owner]),
                "species": np.ascontiguousarray(g["species"][owner].astype(np.int32))}
        real = np.arange(n, dtype=np.int32)
        rho = ref.rho_nmf(full, offs, idx, real)
        plan = residual_pairs(full, owner, image, offs, idx, real)
        kk = np.array([p[0] for p in plan])
        g3 = ref.pt_DV_pairs(full, rho[owner], offs, idx,
                             np.array([p[1] for p in plan], np.int32),
                             np.array([p[2] for p in plan], np.int32))
        Fq = np.zeros((n, 3))
        np.add.at(Fq, kk, g3)
        # the Hessian blocks of evaluate_D2V_i_Dq2_u_MgHx, summed the same way
        h9 = ref.pt_D2V_pairs(full, rho[owner], offs, idx,
                              np.array([p[1] for p in plan], np.int32),
                              np.array([p[2] for p in plan], np.int32))
        H = np.zeros((n, 3, 3))
        np.add.at(H, kk, h9)
        W = ref.pt_DV_dF(full, full["q"], rho[owner], offs, idx, real)
        st = dict(full)
        st["q"] = np.ascontiguousarray(full["q"] * PT_STRETCH)
        rho_s = ref.rho_nmf(st, offs, idx, real)
        W_s = ref.pt_DV_dF(st, full["q"], rho_s[owner], offs, idx, real)
        out.update({f"{name}_rho": rho, f"{name}_Fq": Fq, f"{name}_W": W, f"{name}_H": H,
                    f"{name}_rho_s": rho_s, f"{name}_W_s": W_s})
        # the mean-field stretch derivative (evaluate_DV0_i_dF_bulk_MgHx),
        # sigma and x held, at q0 = q and after the stretch
        mf = dict(full, sigma=np.ascontiguousarray(g["sigma"][owner]))
        W0 = ref.mf_DV0_dF(mf, full["q"], g["rho"][owner], offs, idx, real)
        mfs = dict(mf, q=st["q"])
        rho0_s = ref.mf_rho(mfs, offs, idx, real)
        W0_s = ref.mf_DV0_dF(mfs, full["q"], rho0_s[owner], offs, idx, real)
        out.update({f"{name}_W0": W0, f"{name}_rho0_s": rho0_s, f"{name}_W0_s": W0_s})
        # the mean-field Hessian blocks (evaluate_D2V0_i_Dmeanq2_u_MgHx),
        # summed over i in {u} U N(u) like the gradients
        h9 = ref.mf_D2V0_pairs(mf, g["rho"][owner], offs, idx,
                               np.array([p[1] for p in plan], np.int32),
                               np.array([p[2] for p in plan], np.int32))
        H0 = np.zeros((n, 3, 3))
        np.add.at(H0, kk, h9)
        out[f"{name}_H0"] = H0
        print(f"point forms {name}: {n} sites, {len(plan)} gradient pairs")
    np.savez_compressed(os.path.join(OUT, "point.npz"), **out)


def multipole_fixture():
    """The mean-field forms under the multipole rule (MULTIPOLE_INTEGRAL),
    from the reference built two ways (oracle/Makefile): with its own
    -DNUMERICAL_DERIVATIVES=0, which selects finite-difference Hessians
    (rule 1), and without it, analytic Hessians (rule 2).  On the stored
    topologies of two system fixtures: rho-bar, V0, S0 and the stretch
    derivative evaluate_DV0_i_dF_bulk_MgHx (q0 = q) of every real site, and
    the assembled residuals of a sample of sites."""
    out = {}
    for rule, analytic in ((1, False), (2, True)):
        ref = pyoracle.reference_multipole(analytic)
        if ref is None:
            sys.exit("oracle/_ref/libbtam_ref_mp*.so missing: run `make -C oracle ref` first")
        for name in ("sphere", "ortho_mgh"):
            g = np.load(os.path.join(OUT, f"{name}.npz"))
            n = len(g["x"])
            owner, image, offs, idx = g["owner"], g["image"], g["offs"], g["idx"]
            full = {"q": np.ascontiguousarray(g["q_all"]),
                    "sigma": np.ascontiguousarray(g["sigma"][owner]),
                    "x": np.ascontiguousarray(g["x"][owner]),
                    "species": np.ascontiguousarray(g["species"][owner]),
                    "beta": np.ascontiguousarray(g["beta"][owner]),
                    "gamma": np.ascontiguousarray(g["gamma"][owner])}
            real = np.arange(n, dtype=np.int32)
            rho_real = ref.mf_rho(full, offs, idx, real)
            rho = rho_real[owner]
            us = np.arange(0, n, max(1, n // 40), dtype=np.int32)
            Rq, Rs, Rx = assemble(ref, full, rho, owner, image, offs, idx, us)
            key = f"{name}_r{rule}_"
            out.update({key + "rho": rho_real, key + "V0": ref.V0(full, rho, offs, idx, real),
                        key + "S0": ref.S0(full, rho, offs, idx, real), key + "res_sites": us,
                        key + "Rq": Rq, key + "Rs": Rs, key + "Rx": Rx,
                        key + "W0": ref.mf_DV0_dF(full, full["q"], rho, offs, idx, real)})
            # the assembled Hessian blocks (evaluate_D2V0_i_Dmeanq2_u_MgHx)
            plan = residual_pairs(full, owner, image, offs, idx, real)
            kk = np.array([p_[0] for p_ in plan])
            h9 = ref.mf_D2V0_pairs(full, rho, offs, idx, np.array([p_[1] for p_ in plan], np.int32),
                                   np.array([p_[2] for p_ in plan], np.int32))
            H0 = np.zeros((n, 3, 3))
            np.add.at(H0, kk, h9)
            out[key + "H0"] = H0
            print(f"multipole rule {rule} {name}: {n} real, {len(us)} residual sites")
    np.savez_compressed(os.path.join(OUT, "multipole.npz"), **out)


def pair_plan(owner, image, offs, idx, us):
    """For each u in us, its self entry and every entry p of its list (the
    neighbour ic = idx[p]): (k, entry, uu, o) with entry -1 for the self
    entry and p otherwise, and (uu, o) the argument pair the reference
    evaluates for it: o = owner(ic), uu = u for a real ic, else the image of
    u in o's list with the opposite shift."""
    plan = []
    for k, u in enumerate(us):
        plan.append((k, -1, int(u), int(u)))
        for p in range(offs[u], offs[u + 1]):
            ic = idx[p]
            o = owner[ic]
            T = image[ic]
            uu = int(u)
            if np.any(T != 0):
                uu = -1
                for cand in idx[offs[o]:offs[o + 1]]:
                    if owner[cand] == u and np.all(image[cand] == -T):
                        uu = int(cand)
                        break
                if uu < 0:
                    raise RuntimeError("asymmetric neighbour lists")
            plan.append((k, p, uu, int(o)))
    return plan


def pairs_fixture(ref, orc):
    """The reference's per-pair functions, one (u, i) call at a time, on a
    sample of sites of each system fixture and of a cell with per-site
    temperatures (beta varies from site to site): evaluate_DV0_i_Dq_u_MgHx
    and evaluate_DV0_i_Dxi_u_adp_MgHx (g4, gx), evaluate_DV_i_Dq_u_adp_MgHx
    (pt_g3), evaluate_D2V_i_Dq2_u_MgHx (pt_h9) and
    evaluate_D2V0_i_Dmeanq2_u_MgHx (mf_h9), for the self entry and every
    list entry of each sampled site."""
    out = {}
    systems = {}
    for name in ("sphere", "x5cube", "ortho_mgh", "config1"):
        g = dict(np.load(os.path.join(OUT, f"{name}.npz")))
        systems[name] = g
    # a periodic Mg-H cell whose sites carry temperatures T ~ U[300, 600] K
    hot = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.4, x_range=(0.0, 0.5),
                            sigma_range=(0.08, 0.15), jitter=0.02, seed=9)
    rng = np.random.default_rng(9)
    hot["beta"] = 1.0 / (8.617332478e-5 * rng.uniform(300.0, 600.0, len(hot["x"])))
    full, n, owner, image = pyoracle.expand(hot, orc)
    offs, idx = orc.neighbors(full["q"])
    real = np.arange(n, dtype=np.int32)
    rho_real = ref.mf_rho(full, offs, idx, real)
    us = np.sort(rng.choice(n, 16, replace=False)).astype(np.int32)
    Rq, Rs, Rx = assemble(ref, full, rho_real[owner], owner, image, offs, idx, us)
    g = {k: hot[k] for k in ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell",
                             "periodic")}
    g.update(q_all=full["q"], owner=owner, image=image, offs=offs, idx=idx, rho=rho_real,
             rho_nmf=ref.rho_nmf(full, offs, idx, real), res_sites=us, Rq=Rq, Rs=Rs, Rx=Rx,
             V0=ref.V0(full, rho_real[owner], offs, idx, real))
    systems["hot_cell"] = g
    for name, g in systems.items():
        n = len(g["x"])
        owner, image, offs, idx = g["owner"], g["image"], g["offs"], g["idx"]
        full = {"q": np.ascontiguousarray(g["q_all"]),
                "sigma": np.ascontiguousarray(g["sigma"][owner]),
                "x": np.ascontiguousarray(g["x"][owner]),
                "species": np.ascontiguousarray(g["species"][owner].astype(np.int32))}
        rng = np.random.default_rng(len(name))
        act = np.flatnonzero(g["x"] >= 5e-4)
        pick = [act[g["species"][act] == sp] for sp in (12, 1)]
        us = np.concatenate([rng.choice(p_, min(len(p_), 6), replace=False)
                             for p_ in pick if len(p_)])
        empty = np.flatnonzero(g["x"] < 5e-4)
        if len(empty):
            us = np.append(us, empty[0])  # an empty site: every value is 0
        us = np.sort(us).astype(np.int32)
        plan = pair_plan(owner, image, offs, idx, us)
        uu = np.array([p_[2] for p_ in plan], np.int32)
        oo = np.array([p_[3] for p_ in plan], np.int32)
        g4, gx = ref.DV0_pairs(full, g["rho"][owner], offs, idx, uu, oo)
        pt_g3 = ref.pt_DV_pairs(full, g["rho_nmf"][owner], offs, idx, uu, oo)
        pt_h9 = ref.pt_D2V_pairs(full, g["rho_nmf"][owner], offs, idx, uu, oo)
        mf_h9 = ref.mf_D2V0_pairs(full, g["rho"][owner], offs, idx, uu, oo)
        out.update({f"{name}_us": us,
                    f"{name}_k": np.array([p_[0] for p_ in plan], np.int32),
                    f"{name}_entry": np.array([p_[1] for p_ in plan], np.int32),
                    f"{name}_uu": uu, f"{name}_oo": oo,
                    f"{name}_g4": g4, f"{name}_gx": gx, f"{name}_pt_g3": pt_g3,
                    f"{name}_pt_h9": pt_h9, f"{name}_mf_h9": mf_h9})
        if name == "hot_cell":
            out.update({f"hot_cell_{k}": v for k, v in g.items()})
        # the same pairs under the multipole rule, from the reference built
        # with it (rule 1: the reference's own finite-difference Hessians;
        # rule 2: analytic), at the rule's rho-bar
        if name in ("sphere", "ortho_mgh"):
            for rule, analytic in ((1, False), (2, True)):
                refm = pyoracle.reference_multipole(analytic)
                real = np.arange(n, dtype=np.int32)
                rho_mp = refm.mf_rho(full, offs, idx, real)
                m4, mx = refm.DV0_pairs(full, rho_mp[owner], offs, idx, uu, oo)
                mh = refm.mf_D2V0_pairs(full, rho_mp[owner], offs, idx, uu, oo)
                out.update({f"{name}_mp{rule}_g4": m4, f"{name}_mp{rule}_gx": mx,
                            f"{name}_mp{rule}_h9": mh})
        print(f"pairs {name}: {len(us)} sites, {len(plan)} pairs")
    np.savez_compressed(os.path.join(OUT, "pairs.npz"), **out)


# Slots of the per-term plugin table: (fn, directions) per number of sites;
# fn 0 F, 1 dF_dq, 2 d2F_dq2, 3 dF_dq_FD, 4 d2F_dq2_FD, 5 dF_dn.
TERM_FNS = {2: [(0, [0]), (1, [0, 1]), (2, [0, 1, 2, 3]), (3, [0, 1]), (4, [0, 1, 2, 3]),
                (5, [0, 1])],
            3: [(0, [0]), (1, [0, 1, 2]), (2, list(range(9))), (3, [0, 1, 2]),
                (4, list(range(9))), (5, [0, 1, 2])]}


def termfns_fixture(ref, per=12):
    """Every slot of the reference's per-term plugin table (potential_function:
    F, dF_dq, d2F_dq2, their finite-difference twins and dF_dn) of the four ADP
    terms, each direction, at seeded geometries: sites 1.6-6.5 A from the
    centre (some past the table end), species mixed, occupancies in [0.05, 1]."""
    rng = np.random.default_rng(17)
    rows = []
    for term in range(4):
        ns = 2 if term < 2 else 3
        for fn, dirs in TERM_FNS[ns]:
            for d in dirs:
                for _ in range(per):
                    q = np.zeros(9)
                    q[:3] = rng.uniform(-1.0, 1.0, 3)
                    for k in range(1, ns):
                        v = rng.normal(size=3)
                        q[3 * k:3 * k + 3] = q[:3] + v / np.linalg.norm(v) * rng.uniform(1.6, 6.5)
                    x = rng.uniform(0.05, 1.0, 3)
                    spc = rng.choice([12, 1], 3).astype(np.int32)
                    out = ref.term_eval(term, fn, d, q[:3 * ns], x[:ns], spc[:ns])
                    rows.append((term, fn, d, ns, q, x, spc, out))
    np.savez_compressed(
        os.path.join(OUT, "termfns.npz"),
        meta=np.array([r_[:4] for r_ in rows], np.int32), q=np.array([r_[4] for r_ in rows]),
        x=np.array([r_[5] for r_ in rows]), species=np.array([r_[6] for r_ in rows]),
        out=np.array([r_[7] for r_ in rows]))
    print(f"termfns: {len(rows)} evaluations")


def quad5_fixture(ref, per=8):
    """The reference's 5th-degree rule (Quadrature-Hermitian-5th.cpp) of the
    two pair terms: the average, the averaged gradient of each site and the
    averaged Hessian blocks, at seeded pair geometries (sites 1.6-6.5 A
    apart, widths 0.05-0.2 A, species mixed, occupancies in [0.05, 1])."""
    rng = np.random.default_rng(23)
    rows = []
    for term in (0, 1):
        for mode, dirs in ((0, [0]), (1, [0, 1]), (2, [0, 1, 2, 3])):
            for d in dirs:
                for _ in range(per):
                    q = np.zeros(6)
                    q[:3] = rng.uniform(-1.0, 1.0, 3)
                    v = rng.normal(size=3)
                    q[3:] = q[:3] + v / np.linalg.norm(v) * rng.uniform(1.6, 6.5)
                    sig = rng.uniform(0.05, 0.2, 2)
                    x = rng.uniform(0.05, 1.0, 2)
                    spc = rng.choice([12, 1], 2).astype(np.int32)
                    out = ref.quad5(term, mode, d, q, sig, x, spc)
                    rows.append((term, mode, d, q, sig, x, spc, out))
    np.savez_compressed(
        os.path.join(OUT, "quad5.npz"),
        meta=np.array([r_[:3] for r_ in rows], np.int32), q=np.array([r_[3] for r_ in rows]),
        sigma=np.array([r_[4] for r_ in rows]), x=np.array([r_[5] for r_ in rows]),
        species=np.array([r_[6] for r_ in rows]), out=np.array([r_[7] for r_ in rows]))
    print(f"quad5: {len(rows)} quadratures")


def main():
    ref = pyoracle.reference()
    if ref is not None and sys.argv[1:] == ["--quad5"]:
        quad5_fixture(ref)
        return
    if ref is not None and sys.argv[1:] == ["--termfns"]:
        termfns_fixture(ref)
        return
    if ref is not None and sys.argv[1:] == ["--pairs"]:
        pairs_fixture(ref, pyoracle.Oracle())
        return
    if ref is not None and sys.argv[1:] == ["--point"]:
        point_fixture(ref)
        return
    if sys.argv[1:] == ["--multipole"]:
        multipole_fixture()
        return
    if ref is None:
        sys.exit("oracle/_ref/libbtam_ref.so missing: run `make -C oracle ref` first")
    orc = pyoracle.Oracle()
    # 1. splines of all 13 tables (cubic-spline.cpp:84-128)
    r = np.concatenate([np.linspace(0.0, 7.0, 701), [6.2934034034, 6.29867867868, 6.3, 8.0]])
    F = np.linspace(0.0, 0.2, 201)
    vals = {}
    for t in range(13):
        rr = F if t in (2, 3) else r
        vals[f"t{t}_r"] = rr
        vals[f"t{t}_v"] = np.array([ref.spline(t, v, 0) for v in rr])
        vals[f"t{t}_d"] = np.array([ref.spline(t, v, 1) for v in rr])
    np.savez_compressed(os.path.join(OUT, "splines.npz"), **vals)
    # 2. single-term quadratures: pairs, distinct and coincident triplets
    rng = np.random.default_rng(2024)
    rows = []
    for trial in range(40):
        q = rng.normal(0.0, 2.0, (3, 3))
        q[0] = 0.0
        sig = rng.uniform(0.05, 0.2, 3)
        x = rng.uniform(0.01, 1.0, 3)
        sp = rng.choice([1, 12], 3).astype(np.int32)
        for term in range(4):
            ns = 2 if term < 2 else 3
            for coinc in ([0] if ns == 2 else [0, 1]):
                qq, ss, xx, spc = q.copy(), sig.copy(), x.copy(), sp.copy()
                if coinc:
                    qq[2], ss[2], xx[2], spc[2] = qq[1], ss[1], xx[1], spc[1]
                for mode in range(4):
                    for slot in (range(ns) if mode else [0]):
                        out = np.atleast_1d(ref.quadrature(term, mode, slot, qq[:ns], ss[:ns],
                                                           xx[:ns], spc[:ns], coinc))
                        o3 = np.zeros(3)
                        o3[:len(out)] = out
                        rows.append((term, mode, slot, ns, coinc, qq.ravel(), ss, xx, spc, o3))
    np.savez_compressed(
        os.path.join(OUT, "terms.npz"),
        meta=np.array([r_[:5] for r_ in rows], np.int32),
        q=np.array([r_[5] for r_ in rows]), sigma=np.array([r_[6] for r_ in rows]),
        x=np.array([r_[7] for r_ in rows]), species=np.array([r_[8] for r_ in rows]),
        out=np.array([r_[9] for r_ in rows]))
    print(f"terms: {len(rows)} quadratures")
    # 3. systems
    sphere = lattice.cluster("sphere", 8.0, x_fn=lambda g, rr, n: g.uniform(0.0, 0.6, n),
                             h_fraction=0.5, seed=3)
    system_fixture("sphere", sphere, ref, orc)
    cube = dump.read_dump(os.path.join(REF_TREE, "inputs", "Mg-hcp-cube-x5-x5-x5.dump"))
    system_fixture("x5cube", cube, ref, orc, residual_sample=40, seed=5)
    ortho = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.3, x_range=(0.0, 0.4),
                              sigma_range=(0.08, 0.15), jitter=0.02, seed=5)
    system_fixture("ortho_mgh", ortho, ref, orc)
    system_fixture("config1", lattice.config1(), ref, orc, residual_sample=40, seed=1)
    point_fixture(ref)
    multipole_fixture()
    pairs_fixture(ref, orc)
    termfns_fixture(ref)


if __name__ == "__main__":
    main()
