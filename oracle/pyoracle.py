"""Test infrastructure only: ctypes access to the CPU oracle.

Loads ``oracle/_build/libbtam_oracle.so`` (the restated oracle, always
buildable with g++) and, when present, ``oracle/_ref/libbtam_ref.so`` (the
reference's own arithmetic files compiled unmodified; needs the reference
tree at build time).  Both expose the same per-site entry points with the
prefixes ``orc_`` and ``ref_``.  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libbtam_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbtam_ref.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libbtam_ref_fast.so")
REF_MP_SO = os.path.join(HERE, "_ref", "libbtam_ref_mp.so")
REF_MPA_SO = os.path.join(HERE, "_ref", "libbtam_ref_mpa.so")
TABLES = os.path.join(os.path.dirname(HERE), "bt-am_b200", "data")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


def build_oracle():
    """Compile the restated oracle if it is missing (g++ only)."""
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "_build/libbtam_oracle.so"], cwd=HERE,
                       check=True)
    return ORACLE_SO


class Lib:
    """One of the two CPU libraries (restated oracle or reference build)."""

    def __init__(self, path, prefix, tables=TABLES):
        self.path = path
        self.prefix = prefix
        self.lib = ctypes.CDLL(path)
        f = self._f
        f("spline").restype = ctypes.c_double
        f("spline").argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int]
        f("load_tables").argtypes = [ctypes.c_char_p]
        rc = f("load_tables")(tables.encode())
        if rc != 0:
            raise RuntimeError(f"{path}: cannot load ADP tables from {tables}")

    def _f(self, name):
        return getattr(self.lib, f"{self.prefix}_{name}")

    def spline(self, table, r, deriv=0):
        return self._f("spline")(table, float(r), deriv)

    def quadrature(self, term, mode, slot, q, sigma, x, spc, coincident=0):
        q = np.ascontiguousarray(q, np.float64).ravel()
        sigma = np.ascontiguousarray(sigma, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        spc = np.ascontiguousarray(spc, np.int32)
        out = np.zeros(3)
        self._f("quadrature")(int(term), int(mode), int(slot), len(sigma), int(coincident), _d(q),
                              _d(sigma), _d(x), _i(spc), _d(out))
        return out if mode == 1 else out[0]

    def term_eval(self, term, fn, direction, q, x, spc):
        """One slot of the per-term plugin table at one geometry (reference
        build only: ref_term_eval); 9 values, unused ones 0."""
        q = np.ascontiguousarray(q, np.float64).ravel()
        x = np.ascontiguousarray(x, np.float64)
        spc = np.ascontiguousarray(spc, np.int32)
        out = np.zeros(9)
        rc = self._f("term_eval")(int(term), int(fn), int(direction), len(x), _d(q), _d(x),
                                  _i(spc), _d(out))
        if rc:
            raise ValueError("term_eval")
        return out

    def quad5(self, term, mode, direction, q, sigma, x, spc):
        """The reference's 5th-degree rule over the pair measure of a pair
        term (reference build: ref_quad5; oracle: orc_quad5); 9 values."""
        q = np.ascontiguousarray(q, np.float64).ravel()
        sigma = np.ascontiguousarray(sigma, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        spc = np.ascontiguousarray(spc, np.int32)
        out = np.zeros(9)
        rc = self._f("quad5")(int(term), int(mode), int(direction), _d(q), _d(sigma), _d(x),
                              _i(spc), _d(out))
        if rc:
            raise ValueError("quad5")
        return out

    # --- per-site drivers over a system with CSR neighbour lists ----------
    def mf_rho(self, s, offs, idx, sites):
        sites = np.ascontiguousarray(sites, np.int32)
        out = np.zeros(len(sites))
        self._f("mf_rho")(len(s["x"]), _d(s["q"]), _d(s["sigma"]), _d(s["x"]),
                          _i(s["species"]), _i(offs), _i(idx), _i(sites),
                          len(sites), _d(out))
        return out

    def V0(self, s, rho, offs, idx, sites):
        sites = np.ascontiguousarray(sites, np.int32)
        out = np.zeros(len(sites))
        self._f("V0")(len(s["x"]), _d(s["q"]), _d(s["sigma"]), _d(s["x"]),
                      _i(s["species"]), _d(rho), _i(offs), _i(idx),
                      _i(sites), len(sites), _d(out))
        return out

    def S0(self, s, rho, offs, idx, sites):
        sites = np.ascontiguousarray(sites, np.int32)
        out = np.zeros(len(sites))
        self._f("S0")(len(s["x"]), _d(s["q"]), _d(s["sigma"]), _d(s["x"]),
                      _i(s["species"]), _d(rho), _d(s["beta"]), _d(s["gamma"]),
                      _i(offs), _i(idx), _i(sites), len(sites), _d(out))
        return out

    def DV0_pairs(self, s, rho, offs, idx, u_list, i_list):
        u_list = np.ascontiguousarray(u_list, np.int32)
        i_list = np.ascontiguousarray(i_list, np.int32)
        out4 = np.zeros((len(u_list), 4))
        outx = np.zeros(len(u_list))
        self._f("DV0_pairs")(len(s["x"]), _d(s["q"]), _d(s["sigma"]),
                             _d(s["x"]), _i(s["species"]), _d(rho), _i(offs),
                             _i(idx), _i(u_list), _i(i_list), len(u_list),
                             _d(out4), _d(outx))
        return out4, outx

    def rho_nmf(self, s, offs, idx, sites):
        sites = np.ascontiguousarray(sites, np.int32)
        out = np.zeros(len(sites))
        self._f("rho_nmf")(len(s["x"]), _d(s["q"]), _d(s["x"]),
                           _i(s["species"]), _i(offs), _i(idx), _i(sites),
                           len(sites), _d(out))
        return out


    # --- non-mean-field forms (sigma -> 0) ---------------------------------
    def pt_DV_pairs(self, s, rho, offs, idx, u_list, i_list):
        """dV_i/dq_u per (u, i) pair (evaluate_DV_i_Dq_u_adp_MgHx)."""
        u_list = np.ascontiguousarray(u_list, np.int32)
        i_list = np.ascontiguousarray(i_list, np.int32)
        out = np.zeros((len(u_list), 3))
        self._f("pt_DV_pairs")(len(s["x"]), _d(s["q"]), _d(s["x"]), _i(s["species"]), _d(rho),
                               _i(offs), _i(idx), _i(u_list), _i(i_list), len(u_list), _d(out))
        return out

    def pt_DV_dF(self, s, q0, rho, offs, idx, sites):
        """dV_i/dF per site, 3x3 (evaluate_DV_i_dF_MgHx), reference positions q0."""
        sites = np.ascontiguousarray(sites, np.int32)
        q0 = np.ascontiguousarray(q0, np.float64)
        out = np.zeros((len(sites), 3, 3))
        self._f("pt_DV_dF")(len(s["x"]), _d(s["q"]), _d(q0), _d(s["x"]), _i(s["species"]),
                            _d(rho), _i(offs), _i(idx), _i(sites), len(sites), _d(out))
        return out


    def mf_DV0_dF(self, s, q0, rho, offs, idx, sites):
        """dV0_i/dF per site, 3x3 (evaluate_DV0_i_dF_bulk_MgHx), reference
        positions q0, mean-field density rho of every site."""
        sites = np.ascontiguousarray(sites, np.int32)
        q0 = np.ascontiguousarray(q0, np.float64)
        out = np.zeros((len(sites), 3, 3))
        self._f("mf_DV0_dF")(len(s["x"]), _d(s["q"]), _d(q0), _d(s["sigma"]), _d(s["x"]),
                             _i(s["species"]), _d(rho), _i(offs), _i(idx), _i(sites),
                             len(sites), _d(out))
        return out


    def pt_D2V_pairs(self, s, rho, offs, idx, u_list, i_list):
        """d2V_i/dq_u^2 per (u, i) pair, 3x3 (evaluate_D2V_i_Dq2_u_MgHx)."""
        u_list = np.ascontiguousarray(u_list, np.int32)
        i_list = np.ascontiguousarray(i_list, np.int32)
        out = np.zeros((len(u_list), 3, 3))
        self._f("pt_D2V_pairs")(len(s["x"]), _d(s["q"]), _d(s["x"]), _i(s["species"]),
                                _d(rho), _i(offs), _i(idx), _i(u_list), _i(i_list),
                                len(u_list), _d(out))
        return out


    def mf_D2V0_pairs(self, s, rho, offs, idx, u_list, i_list):
        """d2V0_i/dmean_q_u^2 per (u, i) pair, 3x3
        (evaluate_D2V0_i_Dmeanq2_u_MgHx); rho: mean-field density."""
        u_list = np.ascontiguousarray(u_list, np.int32)
        i_list = np.ascontiguousarray(i_list, np.int32)
        out = np.zeros((len(u_list), 3, 3))
        self._f("mf_D2V0_pairs")(len(s["x"]), _d(s["q"]), _d(s["sigma"]), _d(s["x"]),
                                 _i(s["species"]), _d(rho), _i(offs), _i(idx), _i(u_list),
                                 _i(i_list), len(u_list), _d(out))
        return out


class Oracle(Lib):
    """The restated oracle plus its project-defined pieces."""

    def __init__(self, tables=TABLES):
        super().__init__(build_oracle(), "orc", tables)
        self._f("mass").restype = ctypes.c_double

    def set_rule(self, rule):
        """0: degree-3 Gauss-Hermite rule (the shipped build); 1: multipole
        with finite-difference Hessians (the reference's build flags); 2:
        multipole with analytic Hessians."""
        self._f("set_rule")(int(rule))

    def mass(self, species):
        return self._f("mass")(int(species))

    def ghosts(self, s, rc=6.2934034034, max_ghosts=None):
        n = len(s["x"])
        max_ghosts = max_ghosts or 27 * n
        qg = np.zeros((max_ghosts, 3))
        owner = np.zeros(max_ghosts, np.int32)
        image = np.zeros((max_ghosts, 3), np.int32)
        ng = ctypes.c_int(0)
        cell = np.ascontiguousarray(s["cell"], np.float64)
        origin = np.ascontiguousarray(s["origin"], np.float64)
        per = np.ascontiguousarray(s["periodic"], np.int32)
        rc_ = self._f("ghosts")(n, _d(s["q"]), _d(origin), _d(cell), _i(per),
                                ctypes.c_double(rc), max_ghosts, _d(qg),
                                _i(owner), _i(image), ctypes.byref(ng))
        if rc_ != 0:
            raise RuntimeError(f"orc_ghosts failed with code {rc_}")
        k = ng.value
        return qg[:k].copy(), owner[:k].copy(), image[:k].copy()

    def neighbors(self, q, query=None, rc=6.2934034034, maxn=250):
        q = np.ascontiguousarray(q, np.float64)
        n = len(q)
        query = np.arange(n, dtype=np.int32) if query is None else \
            np.ascontiguousarray(query, np.int32)
        cap = max(1, len(query)) * maxn
        offs = np.zeros(len(query) + 1, np.int32)
        idx = np.zeros(cap, np.int32)
        rc_ = self._f("neighbors")(n, _d(q), ctypes.c_double(rc), maxn,
                                   _i(query), len(query), _i(offs), _i(idx), cap)
        if rc_ != 0:
            raise RuntimeError(f"orc_neighbors failed with code {rc_}")
        return offs, idx[:offs[-1]].copy()

    def residuals(self, s, rho, owner, image, offs, idx, u_list):
        u_list = np.ascontiguousarray(u_list, np.int32)
        nu = len(u_list)
        Rq = np.zeros((nu, 3))
        Rs = np.zeros(nu)
        Rx = np.zeros(nu)
        self._f("residuals")(len(s["x"]), _d(s["q"]), _d(s["sigma"]),
                             _d(s["x"]), _i(s["species"]), _d(s["beta"]),
                             _d(s["gamma"]), _d(rho), _i(owner), _i(image),
                             _i(offs), _i(idx), _i(u_list), nu, _d(Rq),
                             _d(Rs), _d(Rx))
        return Rq, Rs, Rx


def reference(fast=False, tables=TABLES):
    """The reference's own arithmetic (shim build), or None if not built."""
    path = REF_FAST_SO if fast else REF_SO
    if not os.path.exists(path):
        return None
    return Lib(path, "ref", tables)


def reference_multipole(analytic=False, tables=TABLES):
    """The reference built with -DMULTIPOLE_INTEGRAL (and, unless `analytic`,
    its own -DNUMERICAL_DERIVATIVES=0), or None if not built."""
    path = REF_MPA_SO if analytic else REF_MP_SO
    if not os.path.exists(path):
        return None
    return Lib(path, "ref", tables)


def expand(sys_, oracle, rc=6.2934034034):
    """Real sites + periodic images as one site array, with the owner/image
    maps, as the oracle evaluates them.  Returns (all-sites dict, n_real,
    owner, image)."""
    n = len(sys_["x"])
    if any(sys_["periodic"]):
        qg, og, ig = oracle.ghosts(sys_, rc)
    else:
        qg = np.zeros((0, 3))
        og = np.zeros(0, np.int32)
        ig = np.zeros((0, 3), np.int32)
    full = dict(sys_)
    full["q"] = np.ascontiguousarray(np.concatenate([sys_["q"], qg]))
    for k in ("sigma", "x", "beta", "gamma"):
        full[k] = np.ascontiguousarray(np.concatenate([sys_[k], sys_[k][og]]))
    full["species"] = np.ascontiguousarray(
        np.concatenate([sys_["species"], sys_["species"][og]]).astype(np.int32))
    owner = np.concatenate([np.arange(n, dtype=np.int32), og]).astype(np.int32)
    image = np.concatenate([np.zeros((n, 3), np.int32), ig]).astype(np.int32)
    return full, n, np.ascontiguousarray(owner), np.ascontiguousarray(image)


def evaluate(sys_, oracle, sites=None, residual_sites=None, rc=6.2934034034):
    """Full literal evaluation on the real sites of one system: per-site
    mean-field rho, V0 and S0, and the residuals of ``residual_sites``
    (default: all real sites)."""
    full, n, owner, image = expand(sys_, oracle, rc)
    offs, idx = oracle.neighbors(full["q"], rc=rc)
    real = np.arange(n, dtype=np.int32) if sites is None else np.asarray(sites, np.int32)
    rho_real = oracle.mf_rho(full, offs, idx, np.arange(n, dtype=np.int32))
    rho = rho_real[owner]
    V0 = oracle.V0(full, rho, offs, idx, real)
    S0 = oracle.S0(full, rho, offs, idx, real)
    us = real if residual_sites is None else np.asarray(residual_sites, np.int32)
    Rq, Rs, Rx = oracle.residuals(full, rho, owner, image, offs, idx, us)
    return dict(rho=rho_real, V0=V0, S0=S0, Rq=Rq, Rs=Rs, Rx=Rx, offs=offs,
                idx=idx, full=full, owner=owner, image=image, n_real=n)


def sampled_residuals(sys_, oracle, sites, rc=6.2934034034):
    """Literal residuals of a few real sites of a large system.  Neighbour
    lists are built only for the sites the assembly reads (the sampled sites
    and the owners of their neighbours); the other lists stay empty."""
    full, n, owner, image = expand(sys_, oracle, rc)
    sites = np.asarray(sites, np.int32)
    offs_s, idx_s = oracle.neighbors(full["q"], query=sites, rc=rc)
    need = set(int(s) for s in sites)
    for k in range(len(sites)):
        for j in idx_s[offs_s[k]:offs_s[k + 1]]:
            need.add(int(owner[j]))
    query = np.array(sorted(need), np.int32)
    offs_q, idx_q = oracle.neighbors(full["q"], query=query, rc=rc)
    counts = np.zeros(len(full["x"]), np.int64)
    counts[query] = np.diff(offs_q)
    offs = np.zeros(len(full["x"]) + 1, np.int32)
    offs[1:] = np.cumsum(counts)
    idx = np.zeros(offs[-1], np.int32)
    for k, qi in enumerate(query):
        idx[offs[qi]:offs[qi + 1]] = idx_q[offs_q[k]:offs_q[k + 1]]
    rho_q = oracle.mf_rho(full, offs, idx, query)
    rho_real = np.zeros(n)
    rho_real[query] = rho_q
    rho = rho_real[owner]
    V0 = oracle.V0(full, rho, offs, idx, sites)
    Rq, Rs, Rx = oracle.residuals(full, rho, owner, image, offs, idx, sites)
    return dict(rho=rho_real[sites], V0=V0, Rq=Rq, Rs=Rs, Rx=Rx)


def diffusive_graph(q_all, species_all, n_real, rc=2.6, maxn=50):
    """H-H pairs within rc for the real H sites, ascending index, with the
    IEEE distance test sqrt((dx^2 + dy^2) + dz^2) <= rc of the neighbour rule
    (list_of_diffusive_neighs, Neighbors.cpp:139-275); sites without H
    neighbours get empty lists."""
    q_all = np.asarray(q_all)
    h = np.flatnonzero(np.asarray(species_all) == 1)
    offs = np.zeros(n_real + 1, np.int32)
    out = []
    for i in range(n_real):
        lst = []
        if species_all[i] == 1:
            d = q_all[i] - q_all[h]
            r = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
            lst = [int(j) for j in h[(r <= rc) & (h != i)]]
            if len(lst) > maxn:
                raise RuntimeError("more than max_chemical_neighs diffusive neighbours")
        out.extend(lst)
        offs[i + 1] = len(out)
    return offs, np.array(out, np.int32)


def _dmd_args(X, code_all, owner, x_all, beta, mu, moffs, midx, doffs, didx, params):
    arrs = [np.ascontiguousarray(a, np.int32) for a in (code_all, owner)]
    darr = [np.ascontiguousarray(a, np.float64) for a in (x_all, beta, mu)]
    graph = [np.ascontiguousarray(a, np.int32) for a in (moffs, midx, doffs, didx)]
    prm = np.ascontiguousarray(params, np.float64)
    keep = arrs + darr + graph + [prm]
    args = [len(X), _i(arrs[0]), _i(arrs[1]), _d(darr[0]), _d(darr[1]), _d(darr[2]),
            *[_i(a) for a in graph], _d(prm)]
    return args, keep


def dmd_update(oracle, X, code_all, owner, x_all, beta, mu, moffs, midx, doffs, didx, params,
               count_clips=False):
    """One master-equation update of the quanta X (copy returned; with
    count_clips, also the number of edge moves cut to a nonzero room)."""
    X = np.ascontiguousarray(X, np.int64).copy()
    f = oracle.lib.orc_dmd_update
    f.restype = None
    args, keep = _dmd_args(X, code_all, owner, x_all, beta, mu, moffs, midx, doffs, didx,
                           params)
    clipped = ctypes.c_longlong(0)
    f(*args, X.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), ctypes.byref(clipped))
    return (X, clipped.value) if count_clips else X


def dmd_control(oracle, X, code_all, owner, x_all, beta, mu, moffs, midx, doffs, didx, params,
                max_dx):
    """The step-control ratios (edge move over room, site change over
    max_dx) of a step of params[0] at the quanta X."""
    X = np.ascontiguousarray(X, np.int64)
    f = oracle.lib.orc_dmd_control
    f.restype = None
    args, keep = _dmd_args(X, code_all, owner, x_all, beta, mu, moffs, midx, doffs, didx,
                           params)
    out = np.zeros(2)
    f(*args, ctypes.c_double(max_dx), X.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
      _d(out))
    return out


def residuals_on_topology(oracle, real, q_ghost, owner_ghost, image_ghost, offs_real, idx,
                          sites):
    """Literal residuals of `sites` on a given topology: the real-site state
    `real`, the periodic images (positions, owners, shifts) and the
    real-site neighbour lists of a device system, as they stand after a
    relaxation that kept them fixed."""
    n = len(real["x"])
    owner = np.concatenate([np.arange(n), owner_ghost]).astype(np.int32)
    image = np.concatenate([np.zeros((n, 3), np.int32), image_ghost]).astype(np.int32)
    full = dict(real)
    full["q"] = np.ascontiguousarray(np.concatenate([real["q"], q_ghost]))
    for k in ("sigma", "x", "beta", "gamma"):
        full[k] = np.ascontiguousarray(np.asarray(real[k])[owner])
    full["species"] = np.ascontiguousarray(np.asarray(real["species"])[owner].astype(np.int32))
    offs = np.concatenate([offs_real, np.full(len(owner) - n, offs_real[-1])]).astype(np.int32)
    rho_real = oracle.mf_rho(full, offs, idx, np.arange(n, dtype=np.int32))
    rho = rho_real[owner]
    Rq, Rs, Rx = oracle.residuals(full, rho, owner, image, offs, idx, sites)
    return dict(Rq=Rq, Rs=Rs, Rx=Rx)
