"""Python bindings of libbtam.so (the C ABI in include/btam.h).

Thin ctypes wrappers: every call goes to the CUDA library; there is no
Python or CPU implementation of the path.  Importing works without a GPU;
creating tables or systems needs a CUDA device and the built library
(``python bt-am_b200/build.py``), and raises otherwise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libbtam.so")
TABLES_DIR = os.path.join(PKG, "data")
HEADER = os.path.join(os.path.dirname(PKG), "include", "btam.h")

FP64 = 0
FP32C = 1
R_CUTOFF = 6.2934034034
MAXNEIGH = 250
MIN_OCCUPANCY = 5e-4

STATUS = {
    0: "BTAM_OK", 1: "BTAM_ERR_ARG", 2: "BTAM_ERR_IO",
    3: "BTAM_ERR_NEIGHBOR_OVERFLOW", 4: "BTAM_ERR_NO_NEIGHBORS",
    5: "BTAM_ERR_BOX_TOO_SMALL", 6: "BTAM_ERR_NONFINITE", 7: "BTAM_ERR_OOM",
    8: "BTAM_ERR_CUDA", 9: "BTAM_ERR_GHOST_OVERFLOW", 10: "BTAM_ERR_OCCUPANCY",
    11: "BTAM_ERR_SPECIES", 12: "BTAM_ERR_TIMEOUT", 13: "BTAM_ERR_NOT_BUILT",
    14: "BTAM_ERR_OUT_OF_BOX", 15: "BTAM_ERR_TOO_LARGE",
}


class BtamError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: {STATUS.get(code, code)}")


_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_V = ctypes.c_void_p

_PROTOS = {
    "btam_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "btam_version": (ctypes.c_int, []),
    "btam_last_cuda_error": (ctypes.c_char_p, []),
    "btam_pool_usage": (ctypes.c_int, [ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]),
    "btam_tables_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_V)]),
    "btam_tables_destroy": (None, [_V]),
    "btam_tables_mass": (ctypes.c_double, [_V, ctypes.c_int]),
    "btam_tables_spline": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _D, _D, _D]),
    "btam_term_eval": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _D, _D, _I, _D]),
    "btam_term_quadrature": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, _D, _D, _D, _I, _D]),
    "btam_term_quadrature5": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, _D, _D, _D, _I, _D]),
    "btam_system_create": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _I, _D, _D, _D, _D,
                                          _I, ctypes.POINTER(_V)]),
    "btam_system_destroy": (None, [_V]),
    "btam_system_set_state": (ctypes.c_int, [_V, _D, _D, _D]),
    "btam_system_info": (ctypes.c_int, [_V, _I, _I, ctypes.POINTER(ctypes.c_longlong)]),
    "btam_system_stream": (_V, [_V]),
    "btam_neighbors_build": (ctypes.c_int, [_V, ctypes.c_int]),
    "btam_neighbors_copy": (ctypes.c_int, [_V, _I, _I, ctypes.c_longlong]),
    "btam_ghosts_copy": (ctypes.c_int, [_V, _D, _I, _I]),
    "btam_mf_rho": (ctypes.c_int, [_V, ctypes.c_int, _D]),
    "btam_mf_eval": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D]),
    "btam_mf_eval_async": (ctypes.c_int, [_V, ctypes.c_int]),
    "btam_mf_eval_x": (ctypes.c_int, [_V, ctypes.c_int]),
    "btam_mf_eval_state": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D, _D,
                                          _D, _D]),
    "btam_mf_eval_state_async": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D,
                                                _D, _D, _D, ctypes.POINTER(ctypes.c_longlong)]),
    "btam_mf_eval_state_wait": (ctypes.c_int, [_V, ctypes.c_longlong]),
    "btam_results_copy": (ctypes.c_int, [_V, _D, _D, _D, _D, _D, _D, _D]),
    "btam_system_sync": (ctypes.c_int, [_V]),
    "btam_rho_nmf": (ctypes.c_int, [_V, _D]),
    "btam_pt_eval": (ctypes.c_int, [_V, _D, _D, _D, _D, _D]),
    "btam_stretch_apply": (ctypes.c_int, [_V, _D]),
    "btam_pt_hessian": (ctypes.c_int, [_V, _D]),
    "btam_mf_hessian": (ctypes.c_int, [_V, _D]),
    "btam_mf_eval_multipole": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D,
                                              ctypes.POINTER(ctypes.c_double)]),
    "btam_mf_residuals_multipole": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D]),
    "btam_mf_stress_multipole": (ctypes.c_int, [_V, ctypes.c_int, _D, _D]),
    "btam_mf_hessian_multipole": (ctypes.c_int, [_V, ctypes.c_int, _D]),
    "btam_relax_stretch": (ctypes.c_int, [_V, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          _D, _D]),
    "btam_relax_stretch_ngmres": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_int, _D, _D]),
    "btam_relax_stretch_mf": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, _D, _D]),
    "btam_mf_stress": (ctypes.c_int, [_V, ctypes.c_int, _D, _D]),
    "btam_mf_pair_terms": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, ctypes.c_longlong]),
    "btam_mf_pair_terms_multipole": (ctypes.c_int, [_V, ctypes.c_int, _D, _D,
                                                    ctypes.c_longlong]),
    "btam_mf_hessian_pairs": (ctypes.c_int, [_V, _D, _D, ctypes.c_longlong]),
    "btam_mf_hessian_pairs_multipole": (ctypes.c_int, [_V, ctypes.c_int, _D, _D,
                                                       ctypes.c_longlong]),
    "btam_pt_pair_terms": (ctypes.c_int, [_V, _D, _D, _D, _D, ctypes.c_longlong]),
    "btam_mf_eval_profile": (ctypes.c_int, [_V, ctypes.c_int, _D]),
    "btam_probe_fma_peak": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, _D]),
    "btam_probe_gather_peak": (ctypes.c_int, [_V, ctypes.c_double, _D]),
    "btam_autotune": (ctypes.c_int, [_V, ctypes.c_int, _I, _I]),
    "btam_relax": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                  _D, _D]),
    "btam_system_get_state": (ctypes.c_int, [_V, _D, _D, _D]),
    "btam_relax_newton": (ctypes.c_int, [_V, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D,
                                         _D]),
    "btam_dmd_setup": (ctypes.c_int, [_V]),
    "btam_dmd_step": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _D,
                                     ctypes.POINTER(ctypes.c_longlong)]),
    "btam_dmd_step_ctl": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _D,
                                         ctypes.POINTER(ctypes.c_longlong), _D]),
    "btam_dmd_clip_count": (ctypes.c_int, [_V, ctypes.POINTER(ctypes.c_longlong)]),
    "btam_dmd_run": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _D, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_longlong), _D]),
    "btam_dmd_occupancy": (ctypes.c_int, [_V, _D, ctypes.POINTER(ctypes.c_longlong), _D]),
    "btam_dmd_graph_copy": (ctypes.c_int, [_V, _I, _I, ctypes.c_longlong]),
    "btam_batch_create": (ctypes.c_int, [ctypes.POINTER(_V), ctypes.c_int, ctypes.POINTER(_V)]),
    "btam_batch_destroy": (ctypes.c_int, [_V]),
    "btam_batch_info": (ctypes.c_int, [_V, _I, _I, _I, ctypes.POINTER(ctypes.c_longlong)]),
    "btam_batch_stream": (_V, [_V]),
    "btam_batch_set_state": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D]),
    "btam_batch_autotune": (ctypes.c_int, [_V, ctypes.c_int, _I, _I]),
    "btam_batch_set_variants": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "btam_set_variants": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "btam_batch_eval_async": (ctypes.c_int, [_V, ctypes.c_int]),
    "btam_batch_sync": (ctypes.c_int, [_V]),
    "btam_batch_results_copy": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D]),
    "btam_batch_totals_copy": (ctypes.c_int, [_V, _D]),
    "btam_estimate_bytes": (ctypes.c_longlong, [ctypes.c_int, _D, _I]),
    "btam_server_create": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_longlong,
                                          ctypes.POINTER(_V)]),
    "btam_server_submit": (ctypes.c_int, [_V, _V, ctypes.POINTER(ctypes.c_longlong)]),
    "btam_server_wait": (ctypes.c_int, [_V, ctypes.c_longlong, ctypes.c_double, _V, _D, _D, _D]),
    "btam_server_stats": (ctypes.c_int, [_V, ctypes.POINTER(ctypes.c_longlong), _I,
                                         ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong)]),
    "btam_server_destroy": (ctypes.c_int, [_V]),
    "btam_server_batch_stats": (ctypes.c_int, [_V, ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.POINTER(ctypes.c_longlong)]),
    "btam_mf_eval_noalloc": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _V, _V, _V, _V,
                                            _V, _V, _V, _V, _V, _V, _V, _V, _V]),
}



class JobSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("precision", ctypes.c_int), ("mode", ctypes.c_int),
                ("n", ctypes.c_int), ("q", _D), ("sigma", _D), ("x", _D), ("species", _I),
                ("beta", _D), ("gamma", _D), ("origin", _D), ("cell", _D), ("periodic", _I),
                ("tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("lbfgs_m", ctypes.c_int),
                ("sigma_min", ctypes.c_double), ("sigma_max", ctypes.c_double),
                ("x_min", ctypes.c_double), ("nsteps", ctypes.c_int),
                ("dmd_params", ctypes.c_double * 5), ("plain", ctypes.c_int)]


class JobResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("kind", ctypes.c_int), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_start", ctypes.c_double),
                ("t_end", ctypes.c_double), ("norm", ctypes.c_double),
                ("objective", ctypes.c_double), ("iterations", ctypes.c_int),
                ("evaluations", ctypes.c_int), ("converged", ctypes.c_int),
                ("h_quanta_hi", ctypes.c_longlong), ("h_quanta_lo", ctypes.c_longlong)]


_lib = None


def lib():
    """The loaded CUDA library.  Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with "
                               "`python bt-am_b200/build.py` (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names declared in include/btam.h (for the symbol-export test)."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(btam_[a-z0-9_]+)\s*\(", text)))


def _d(a):
    return None if a is None else a.ctypes.data_as(_D)


def _i(a):
    return None if a is None else a.ctypes.data_as(_I)


def _check(code, what):
    if code != 0:
        if code in (7, 8):  # BTAM_ERR_OOM, BTAM_ERR_CUDA: name the runtime error
            name = lib().btam_last_cuda_error().decode()
            if name:
                what = f"{what} ({name})"
        raise BtamError(code, what)


def probe_gather_peak(tables, seconds=0.5):
    """Random 32-byte record gathers from the L1-resident spline tables,
    GB/s over the device."""
    out = np.zeros(1)
    _check(lib().btam_probe_gather_peak(tables.handle, float(seconds), _d(out)),
           "btam_probe_gather_peak")
    return float(out[0])


def probe_fma_peak(fp64=False, seconds=0.5):
    """Measured FMA throughput (TFLOP/s) of the current device."""
    out = np.zeros(1)
    _check(lib().btam_probe_fma_peak(int(fp64), float(seconds), _d(out)),
           "btam_probe_fma_peak")
    return float(out[0])


def pool_usage():
    """(used, reserved) bytes of the library's device-memory pool on the
    current device."""
    used, reserved = ctypes.c_longlong(0), ctypes.c_longlong(0)
    _check(lib().btam_pool_usage(ctypes.byref(used), ctypes.byref(reserved)), "btam_pool_usage")
    return used.value, reserved.value


class Tables:
    """The ADP tables on the device (init_adp_MgHx for MgMg, HH and MgH)."""

    def __init__(self, directory=TABLES_DIR):
        h = _V()
        _check(lib().btam_tables_load(directory.encode(), ctypes.byref(h)),
               "btam_tables_load")
        self.handle = h

    def mass(self, species):
        return lib().btam_tables_mass(self.handle, int(species))

    def spline(self, table, r):
        r = np.ascontiguousarray(r, np.float64)
        v = np.zeros_like(r)
        dv = np.zeros_like(r)
        _check(lib().btam_tables_spline(self.handle, table, len(r), _d(r), _d(v), _d(dv)),
               "btam_tables_spline")
        return v, dv

    def term(self, term, fn, direction, q, x, species):
        """One slot of the per-term plugin table (potential_function) at n
        geometries: term 0 rho_ij, 1 V_pair_ij, 2 V_dipole_ij1j2,
        3 V_quadrupole_ij1j2; fn 0 F, 1 dF_dq, 2 d2F_dq2, 3 dF_dq_FD,
        4 d2F_dq2_FD, 5 dF_dn.  q (n, 9), x and species (n, 3); returns
        (n, 9), the slot's values first."""
        q = np.ascontiguousarray(np.asarray(q, np.float64).reshape(-1, 9))
        x = np.ascontiguousarray(np.asarray(x, np.float64).reshape(-1, 3))
        sp = np.ascontiguousarray(np.asarray(species, np.int32).reshape(-1, 3))
        n = len(q)
        if len(x) != n or len(sp) != n:
            raise ValueError("q, x and species need one row per geometry")
        out = np.zeros((n, 9))
        _check(lib().btam_term_eval(self.handle, int(term), int(fn), int(direction), n, _d(q),
                                    _d(x), _i(sp), _d(out)), "btam_term_eval")
        return out

    def term_quadrature(self, term, mode, slot, q, sigma, x, species, coincident=False):
        """A term averaged over the mean-field measure with the degree-3
        rule: mode 0 the value, 1 d/d mean q of slot (3 values), 2 d/d
        sigma of slot, 3 d/dx of slot.  Returns (n, 9), the values first."""
        q = np.ascontiguousarray(np.asarray(q, np.float64).reshape(-1, 9))
        sg = np.ascontiguousarray(np.asarray(sigma, np.float64).reshape(-1, 3))
        x = np.ascontiguousarray(np.asarray(x, np.float64).reshape(-1, 3))
        sp = np.ascontiguousarray(np.asarray(species, np.int32).reshape(-1, 3))
        n = len(q)
        if len(sg) != n or len(x) != n or len(sp) != n:
            raise ValueError("q, sigma, x and species need one row per geometry")
        out = np.zeros((n, 9))
        _check(lib().btam_term_quadrature(self.handle, int(term), int(mode), int(slot),
                                          int(bool(coincident)), n, _d(q), _d(sg), _d(x),
                                          _i(sp), _d(out)), "btam_term_quadrature")
        return out

    def term_quadrature5(self, term, mode, direction, q, sigma, x, species):
        """The 5th-degree rule over the pair measure of a pair term: mode 0
        the average of F, 1 of dF_dq(direction), 2 of d2F_dq2(direction).
        q (n, 6), sigma, x, species (n, 2); returns (n, 9)."""
        n = len(q)
        qq = np.zeros((n, 9))
        qq[:, :6] = np.asarray(q, np.float64).reshape(n, 6)
        pad = lambda v, dt: np.ascontiguousarray(
            np.pad(np.asarray(v, dt).reshape(n, 2), ((0, 0), (0, 1))))
        sg, x, sp = pad(sigma, np.float64), pad(x, np.float64), pad(species, np.int32)
        out = np.zeros((n, 9))
        _check(lib().btam_term_quadrature5(self.handle, int(term), int(mode), int(direction), n,
                                           _d(qq), _d(sg), _d(x), _i(sp), _d(out)),
               "btam_term_quadrature5")
        return out

    def close(self):
        if self.handle:
            lib().btam_tables_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class System:
    """One device-resident system (the reference's DMSwarm of sites)."""

    def __init__(self, tables, sysdict):
        s = sysdict
        self.tables = tables
        self.n = len(s["x"])
        q = np.ascontiguousarray(s["q"], np.float64)
        sigma = np.ascontiguousarray(s["sigma"], np.float64)
        x = np.ascontiguousarray(s["x"], np.float64)
        spc = np.ascontiguousarray(s["species"], np.int32)
        beta = np.ascontiguousarray(s.get("beta"), np.float64) if s.get("beta") is not None else None
        gamma = np.ascontiguousarray(s.get("gamma"), np.float64) if s.get("gamma") is not None else None
        origin = np.ascontiguousarray(s["origin"], np.float64)
        cell = np.ascontiguousarray(s["cell"], np.float64).reshape(9)
        per = np.ascontiguousarray(s["periodic"], np.int32)
        h = _V()
        _check(lib().btam_system_create(tables.handle, self.n, _d(q), _d(sigma), _d(x),
                                        _i(spc), _d(beta), _d(gamma), _d(origin), _d(cell),
                                        _i(per), ctypes.byref(h)), "btam_system_create")
        self.handle = h
        self.all_sites = None
        self._inflight = {}  # evaluate_state_async tickets -> their arrays

    # -- state and topology
    def set_state(self, q=None, sigma=None, x=None):
        q = None if q is None else np.ascontiguousarray(q, np.float64)
        sigma = None if sigma is None else np.ascontiguousarray(sigma, np.float64)
        x = None if x is None else np.ascontiguousarray(x, np.float64)
        _check(lib().btam_system_set_state(self.handle, _d(q), _d(sigma), _d(x)),
               "btam_system_set_state")

    def build_neighbors(self, all_sites=False):
        _check(lib().btam_neighbors_build(self.handle, int(bool(all_sites))),
               "btam_neighbors_build")
        self.all_sites = bool(all_sites)

    def info(self):
        nr, ng, npairs = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        _check(lib().btam_system_info(self.handle, ctypes.byref(nr), ctypes.byref(ng),
                                      ctypes.byref(npairs)), "btam_system_info")
        return nr.value, ng.value, npairs.value

    def neighbors(self):
        nr, ng, npairs = self.info()
        n_list = nr + ng if self.all_sites else nr
        offs = np.zeros(n_list + 1, np.int32)
        idx = np.zeros(max(npairs, 1), np.int32)
        _check(lib().btam_neighbors_copy(self.handle, _i(offs), _i(idx), len(idx)),
               "btam_neighbors_copy")
        return offs, idx[:npairs]

    def ghosts(self):
        nr, ng, _ = self.info()
        q = np.zeros((ng, 3))
        owner = np.zeros(ng, np.int32)
        image = np.zeros((ng, 3), np.int32)
        if ng:
            _check(lib().btam_ghosts_copy(self.handle, _d(q), _i(owner), _i(image)),
                   "btam_ghosts_copy")
        return q, owner, image

    @property
    def stream(self):
        return lib().btam_system_stream(self.handle)

    # -- evaluation
    def mf_rho(self, precision=FP64):
        out = np.zeros(self.n)
        _check(lib().btam_mf_rho(self.handle, precision, _d(out)), "btam_mf_rho")
        return out

    def evaluate(self, precision=FP64):
        n = self.n
        out = dict(rho=np.zeros(n), V0=np.zeros(n), S0=np.zeros(n), Rq=np.zeros((n, 3)),
                   Rs=np.zeros(n), Rx=np.zeros(n), totals=np.zeros(4))
        _check(lib().btam_mf_eval(self.handle, precision, _d(out["rho"]), _d(out["V0"]),
                                  _d(out["S0"]), _d(out["Rq"]), _d(out["Rs"]), _d(out["Rx"]),
                                  _d(out["totals"])), "btam_mf_eval")
        return out

    def evaluate_state(self, precision=FP64, q=None, sigma=None, x=None):
        """New state and its evaluation in one call (btam_mf_eval_state)."""
        n = self.n
        out = dict(rho=np.zeros(n), V0=np.zeros(n), S0=np.zeros(n), Rq=np.zeros((n, 3)),
                   Rs=np.zeros(n), Rx=np.zeros(n), totals=np.zeros(4))
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        q, sigma, x = cv(q), cv(sigma), cv(x)
        _check(lib().btam_mf_eval_state(self.handle, precision, _d(q), _d(sigma), _d(x),
                                        _d(out["rho"]), _d(out["V0"]), _d(out["S0"]),
                                        _d(out["Rq"]), _d(out["Rs"]), _d(out["Rx"]),
                                        _d(out["totals"])), "btam_mf_eval_state")
        return out

    def evaluate_state_async(self, precision=FP64, q=None, sigma=None, x=None, out=None):
        """btam_mf_eval_state_async: enqueues the new state, its evaluation
        and the copies of the results into `out` (a dict of float64 arrays
        named as evaluate_state's; pin them for overlapped copies) and
        returns a ticket for wait_state.  The arrays (inputs included) must
        stay alive and untouched until then."""
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        q, sigma, x = cv(q), cv(sigma), cv(x)
        out = out or {}
        for k, v in out.items():
            assert v.dtype == np.float64 and v.flags["C_CONTIGUOUS"], k
        tk = ctypes.c_longlong()
        args = [_d(out.get(k)) for k in ("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals")]
        _check(lib().btam_mf_eval_state_async(self.handle, precision, _d(q), _d(sigma), _d(x),
                                              *args, ctypes.byref(tk)),
               "btam_mf_eval_state_async")
        self._inflight[tk.value] = (q, sigma, x, out)  # kept alive until the wait
        return tk.value

    def wait_state(self, ticket):
        """Waits for a btam_mf_eval_state_async call; raises on its status."""
        keep = self._inflight.pop(ticket, None)
        _check(lib().btam_mf_eval_state_wait(self.handle, int(ticket)), "btam_mf_eval_state_wait")
        return keep[3] if keep else None

    def evaluate_async(self, precision=FP64):
        _check(lib().btam_mf_eval_async(self.handle, precision), "btam_mf_eval_async")

    def evaluate_x(self, precision=FP64):
        """The occupancy gradients alone (btam_mf_eval_x): rho, V0, S0, Rx and
        totals of the state, Rq and Rs 0; synchronises."""
        _check(lib().btam_mf_eval_x(self.handle, precision), "btam_mf_eval_x")
        return self.results(want=("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals"))

    def sync(self):
        _check(lib().btam_system_sync(self.handle), "btam_system_sync")

    def results(self, want=("V0", "Rq", "Rs", "Rx", "totals")):
        n = self.n
        shapes = dict(rho=(n,), V0=(n,), S0=(n,), Rq=(n, 3), Rs=(n,), Rx=(n,), totals=(4,))
        out = {k: np.zeros(shapes[k]) for k in want}
        args = [_d(out.get(k)) for k in ("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals")]
        _check(lib().btam_results_copy(self.handle, *args), "btam_results_copy")
        return out

    def get_state(self):
        q = np.zeros((self.n, 3))
        sigma = np.zeros(self.n)
        x = np.zeros(self.n)
        _check(lib().btam_system_get_state(self.handle, _d(q), _d(sigma), _d(x)),
               "btam_system_get_state")
        return q, sigma, x

    # -- consumers: relaxation and the hydrogen master equation
    def relax(self, mode=0, tol=1e-8, max_iter=500, m=8, sigma_min=0.001, sigma_max=0.4,
              x_min=0.01):
        """Relaxation of (q, sigma) on the device: L-BFGS (modes 0-2, m pairs)
        or N-GMRES(m) with the critical-point line search (mode 4).  Returns a
        dict with the final projected residual norm, iterations, evaluations,
        objective and status (1 converged, 0 iteration limit, -1 stalled)."""
        info = np.zeros(5)
        bd = np.array([sigma_min, sigma_max, x_min], np.float64)
        _check(lib().btam_relax(self.handle, mode, tol, max_iter, m, _d(bd), _d(info)),
               "btam_relax")
        return dict(norm=info[0], iterations=int(info[1]), evaluations=int(info[2]),
                    objective=info[3], status=int(info[4]))

    def relax_newton(self, tol=1e-8, max_newton=50, max_cg=200, sigma_min=0.001,
                     sigma_max=0.4, x_min=0.01):
        """Damped truncated-Newton relaxation of (q, sigma) (FP64,
        Hessian-vector products by differences of the residual).  Returns a
        dict like relax() plus the CG iteration count."""
        info = np.zeros(6)
        bd = np.array([sigma_min, sigma_max, x_min], np.float64)
        _check(lib().btam_relax_newton(self.handle, tol, max_newton, max_cg, _d(bd), _d(info)),
               "btam_relax_newton")
        return dict(norm=info[0], iterations=int(info[1]), evaluations=int(info[2]),
                    objective=info[3], status=int(info[4]), cg_iterations=int(info[5]))

    def dmd_setup(self):
        _check(lib().btam_dmd_setup(self.handle), "btam_dmd_setup")

    def dmd_step(self, nsteps=1, precision=FP64, dt=4e-4, Df=0.045, dr=3.2, min_dx=1e-8,
                 max_x=0.9):
        """Master-equation steps; returns the exact total of the occupancy
        quanta (Python int, units of 2^-50)."""
        prm = np.array([dt, Df, dr, min_dx, max_x], np.float64)
        tot = (ctypes.c_longlong * 2)()
        _check(lib().btam_dmd_step(self.handle, precision, nsteps, _d(prm), tot),
               "btam_dmd_step")
        hi, lo = tot[0], tot[1] & 0xFFFFFFFFFFFFFFFF
        return (hi << 64) + lo

    def dmd_step_ctl(self, nsteps=1, precision=FP64, dt=4e-4, Df=0.045, dr=3.2, min_dx=1e-8,
                     max_x=0.9, max_dx=0.05, max_sub=64):
        """Master-equation steps with step control; returns (total quanta,
        stats dict: substeps, subdivided, clipped, worst_ratio)."""
        prm = np.array([dt, Df, dr, min_dx, max_x, max_dx, max_sub], np.float64)
        tot = (ctypes.c_longlong * 2)()
        st = np.zeros(4)
        _check(lib().btam_dmd_step_ctl(self.handle, precision, nsteps, _d(prm), tot, _d(st)),
               "btam_dmd_step_ctl")
        hi, lo = tot[0], tot[1] & 0xFFFFFFFFFFFFFFFF
        return (hi << 64) + lo, dict(substeps=int(st[0]), subdivided=int(st[1]),
                                     clipped=int(st[2]), worst_ratio=float(st[3]))

    def dmd_run(self, nsteps, precision=FP64, relax_every=0, relax_mode=0, relax_tol=1e-6,
                relax_max_iter=200, dt=4e-4, Df=0.045, dr=3.2, min_dx=1e-8, max_x=0.9,
                max_dx=0.05, max_sub=64):
        """Controlled master-equation steps with a (q, sigma) relaxation every
        relax_every steps; returns (total quanta, stats dict)."""
        prm = np.array([dt, Df, dr, min_dx, max_x, max_dx, max_sub], np.float64)
        tot = (ctypes.c_longlong * 2)()
        st = np.zeros(6)
        _check(lib().btam_dmd_run(self.handle, precision, nsteps, _d(prm), relax_every,
                                  relax_mode, relax_tol, relax_max_iter, tot, _d(st)),
               "btam_dmd_run")
        hi, lo = tot[0], tot[1] & 0xFFFFFFFFFFFFFFFF
        return (hi << 64) + lo, dict(substeps=int(st[0]), subdivided=int(st[1]),
                                     clipped=int(st[2]), worst_ratio=float(st[3]),
                                     relaxations=int(st[4]), relax_evaluations=int(st[5]))

    def dmd_clip_count(self):
        c = ctypes.c_longlong(0)
        _check(lib().btam_dmd_clip_count(self.handle, ctypes.byref(c)), "btam_dmd_clip_count")
        return c.value

    def dmd_occupancy(self):
        x = np.zeros(self.n)
        qn = np.zeros(self.n, np.int64)
        mu = np.zeros(self.n)
        _check(lib().btam_dmd_occupancy(self.handle, _d(x),
                                        qn.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                        _d(mu)), "btam_dmd_occupancy")
        return x, qn, mu

    def dmd_graph(self):
        offs = np.zeros(self.n + 1, np.int32)
        _check(lib().btam_dmd_graph_copy(self.handle, _i(offs), None, 0), "btam_dmd_graph_copy")
        idx = np.zeros(max(int(offs[-1]), 1), np.int32)
        _check(lib().btam_dmd_graph_copy(self.handle, _i(offs), _i(idx), len(idx)),
               "btam_dmd_graph_copy")
        return offs, idx[:offs[-1]]

    def autotune(self, precision=FP32C):
        """Pick the fastest kernel shapes for this system; returns their
        indices (pass 1, pass 2)."""
        v1, v2 = ctypes.c_int(), ctypes.c_int()
        _check(lib().btam_autotune(self.handle, precision, ctypes.byref(v1), ctypes.byref(v2)),
               "btam_autotune")
        return v1.value, v2.value

    def set_variants(self, precision, v1, v2):
        """Pins the launch variants (as returned by autotune)."""
        _check(lib().btam_set_variants(self.handle, precision, int(v1), int(v2)),
               "btam_set_variants")

    def profile(self, precision=FP64):
        """Per-kernel device times (ms) of one evaluation: pass-1 pair-rule
        kernel, pass-1 site kernel, pass-2 pair kernel, pass-2 site kernel,
        totals (the pair kernels read ~0 for the directed variants)."""
        ms = np.zeros(5)
        _check(lib().btam_mf_eval_profile(self.handle, precision, _d(ms)),
               "btam_mf_eval_profile")
        return ms

    def rho_nmf(self):
        out = np.zeros(self.n)
        _check(lib().btam_rho_nmf(self.handle, _d(out)), "btam_rho_nmf")
        return out

    # -- non-mean-field forms and the bulk stretch relaxation
    def pt_eval(self):
        """Non-mean-field forms at the current q and x: dict of rho (n), V (n),
        Fq (n, 3) = sum_{i in {u} U N(u)} dV_i/dq_u, W (n, 3, 3) = dV_u/dF at
        q0 = q, totals (12): sum V, sum |Fq|^2, sum W (9), 0."""
        n = self.n
        out = dict(rho=np.zeros(n), V=np.zeros(n), Fq=np.zeros((n, 3)), W=np.zeros((n, 3, 3)),
                   totals=np.zeros(12))
        _check(lib().btam_pt_eval(self.handle, _d(out["rho"]), _d(out["V"]), _d(out["Fq"]),
                                  _d(out["W"]), _d(out["totals"])), "btam_pt_eval")
        return out

    def pt_hessian(self):
        """Hessian blocks of the non-mean-field forms, (n, 3, 3): the sum over
        i in {u} U N(u) of evaluate_D2V_i_Dq2_u_MgHx."""
        H = np.zeros((self.n, 3, 3))
        _check(lib().btam_pt_hessian(self.handle, _d(H)), "btam_pt_hessian")
        return H

    def mf_eval_multipole(self, rule=1):
        """rho-bar, V0 per site and their sum under the multipole rule
        (MULTIPOLE_INTEGRAL): rule MP_FD (1) with the finite-difference
        Hessians of the reference's build flags, MP_ANALYTIC (2) with
        analytic Hessians.  FP64.  The per-site S0 of the same call is kept
        in `last_S0`."""
        rho = np.zeros(self.n)
        V0 = np.zeros(self.n)
        S0 = np.zeros(self.n)
        E = ctypes.c_double(0.0)
        _check(lib().btam_mf_eval_multipole(self.handle, int(rule), _d(rho), _d(V0), _d(S0),
                                            ctypes.byref(E)), "btam_mf_eval_multipole")
        self.last_S0 = S0
        return rho, V0, E.value

    def mf_residuals_multipole(self, rule=1):
        """(Rq (n, 3), Rs (n,), Rx (n,)) under the multipole rule, FP64."""
        Rq = np.zeros((self.n, 3))
        Rs = np.zeros(self.n)
        Rx = np.zeros(self.n)
        _check(lib().btam_mf_residuals_multipole(self.handle, int(rule), _d(Rq), _d(Rs), _d(Rx)),
               "btam_mf_residuals_multipole")
        return Rq, Rs, Rx

    def mf_stress_multipole(self, rule=1):
        """(W0 (n, 3, 3), total (3, 3)): evaluate_DV0_i_dF_bulk_MgHx under
        the multipole rule at q0 = q, FP64."""
        W = np.zeros((self.n, 3, 3))
        tot = np.zeros((3, 3))
        _check(lib().btam_mf_stress_multipole(self.handle, int(rule), _d(W), _d(tot)),
               "btam_mf_stress_multipole")
        return W, tot

    def mf_hessian_multipole(self, rule=1):
        """Mean-field Hessian blocks (n, 3, 3) under the multipole rule."""
        H = np.zeros((self.n, 3, 3))
        _check(lib().btam_mf_hessian_multipole(self.handle, int(rule), _d(H)),
               "btam_mf_hessian_multipole")
        return H

    def mf_hessian(self):
        """Mean-field Hessian blocks, (n, 3, 3): the sum over i in {u} U N(u)
        of evaluate_D2V0_i_Dmeanq2_u_MgHx (FP64)."""
        H = np.zeros((self.n, 3, 3))
        _check(lib().btam_mf_hessian(self.handle, _d(H)), "btam_mf_hessian")
        return H

    def stretch(self, F):
        """q <- diag(F) q, cell and origin likewise; neighbour lists kept."""
        F = np.ascontiguousarray(F, np.float64)
        _check(lib().btam_stretch_apply(self.handle, _d(F)), "btam_stretch_apply")

    def relax_stretch(self, atol=1e-12, rtol=1e-10, max_iter=20, F0=(1.0, 1.0, 1.0)):
        """Bulk stretch relaxation (diagonal F zeroing the mean stress of the
        non-mean-field forms); leaves the system stretched.  Returns (F, info
        dict: norm, iterations, evaluations, status, volume)."""
        F = np.ascontiguousarray(F0, np.float64).copy()
        info = np.zeros(5)
        _check(lib().btam_relax_stretch(self.handle, atol, rtol, max_iter, _d(F), _d(info)),
               "btam_relax_stretch")
        return F, dict(norm=info[0], iterations=int(info[1]), evaluations=int(info[2]),
                       status=int(info[3]), volume=info[4])

    def relax_stretch_ngmres(self, m=3, atol=1e-12, rtol=1e-10, max_iter=50,
                             F0=(1.0, 1.0, 1.0)):
        """The same relaxation with N-GMRES(m) and the critical-point line
        search, the reference's configured solver.  Returns (F, info)."""
        F = np.ascontiguousarray(F0, np.float64).copy()
        info = np.zeros(5)
        _check(lib().btam_relax_stretch_ngmres(self.handle, int(m), atol, rtol, max_iter, _d(F),
                                               _d(info)), "btam_relax_stretch_ngmres")
        return F, dict(norm=info[0], iterations=int(info[1]), evaluations=int(info[2]),
                       status=int(info[3]), volume=info[4])

    def mf_stress(self, precision=FP64):
        """Mean-field stress dV0_u/dF at q0 = q, sigma and x held: (per-site
        (n, 3, 3), sum (3, 3))."""
        W = np.zeros((self.n, 3, 3))
        tot = np.zeros(9)
        _check(lib().btam_mf_stress(self.handle, precision, _d(W), _d(tot)), "btam_mf_stress")
        return W, tot.reshape(3, 3)

    def pair_terms(self, precision=FP64):
        """Unweighted per-pair terms of the residual assembly: (self (n, 5):
        dV0_u/d(q_u, sigma_u, x_u); slot (entries, 5): dV0_j/d(q_u, sigma_u,
        x_u) for every entry (u, j) of the real sites' neighbour lists)."""
        offs, _ = self.neighbors()
        n_slots = int(offs[self.n])
        selfv = np.zeros((self.n, 5))
        slot = np.zeros((max(n_slots, 1), 5))
        _check(lib().btam_mf_pair_terms(self.handle, precision, _d(selfv), _d(slot), n_slots),
               "btam_mf_pair_terms")
        return selfv, slot[:n_slots]

    def _n_slots(self):
        offs, _ = self.neighbors()
        return int(offs[self.n])

    def pair_terms_multipole(self, rule=1):
        """Per-pair terms under the multipole rule (as pair_terms)."""
        ns = self._n_slots()
        selfv, slot = np.zeros((self.n, 5)), np.zeros((max(ns, 1), 5))
        _check(lib().btam_mf_pair_terms_multipole(self.handle, rule, _d(selfv), _d(slot), ns),
               "btam_mf_pair_terms_multipole")
        return selfv, slot[:ns]

    def mf_hessian_pairs(self, rule=0):
        """Per-pair mean-field Hessian blocks (rule 0: degree-3; 1, 2: the
        multipole rule): (Hself (n, 3, 3), Hslot (entries, 3, 3))."""
        ns = self._n_slots()
        Hs, Hp = np.zeros((self.n, 3, 3)), np.zeros((max(ns, 1), 3, 3))
        if rule:
            code = lib().btam_mf_hessian_pairs_multipole(self.handle, rule, _d(Hs), _d(Hp), ns)
        else:
            code = lib().btam_mf_hessian_pairs(self.handle, _d(Hs), _d(Hp), ns)
        _check(code, "btam_mf_hessian_pairs")
        return Hs, Hp[:ns]

    def pt_pair_terms(self):
        """Per-pair non-mean-field terms: (self3 (n, 3), slot3 (entries, 3),
        Hself (n, 3, 3), Hslot (entries, 3, 3))."""
        ns = self._n_slots()
        g, gp = np.zeros((self.n, 3)), np.zeros((max(ns, 1), 3))
        Hs, Hp = np.zeros((self.n, 3, 3)), np.zeros((max(ns, 1), 3, 3))
        _check(lib().btam_pt_pair_terms(self.handle, _d(g), _d(gp), _d(Hs), _d(Hp), ns),
               "btam_pt_pair_terms")
        return g, gp[:ns], Hs, Hp[:ns]

    def relax_stretch_mf(self, precision=FP64, atol=1e-12, rtol=1e-10, max_iter=20,
                         F0=(1.0, 1.0, 1.0)):
        """Bulk stretch relaxation on the mean-field stress (sigma, x held)."""
        F = np.ascontiguousarray(F0, np.float64).copy()
        info = np.zeros(5)
        _check(lib().btam_relax_stretch_mf(self.handle, precision, atol, rtol, max_iter, _d(F),
                                           _d(info)), "btam_relax_stretch_mf")
        return F, dict(norm=info[0], iterations=int(info[1]), evaluations=int(info[2]),
                       status=int(info[3]), volume=info[4])

    def close(self):
        if getattr(self, "handle", None):
            lib().btam_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many built systems evaluated together: one CUDA graph launch (pass 1,
    pass 2, per-system totals) per evaluation of all of them.  The systems
    must stay alive while the batch is used."""

    def __init__(self, systems):
        self.systems = list(systems)
        arr = (_V * len(self.systems))(*[s.handle for s in self.systems])
        h = _V()
        _check(lib().btam_batch_create(arr, len(self.systems), ctypes.byref(h)),
               "btam_batch_create")
        self.handle = h

    def info(self):
        ns, nr, na = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        npairs = ctypes.c_longlong()
        _check(lib().btam_batch_info(self.handle, ctypes.byref(ns), ctypes.byref(nr),
                                     ctypes.byref(na), ctypes.byref(npairs)), "btam_batch_info")
        return dict(n_sys=ns.value, n_real=nr.value, n_all=na.value, n_pairs=npairs.value)

    def stream(self):
        return lib().btam_batch_stream(self.handle)

    def set_state(self, k, q=None, sigma=None, x=None):
        q = None if q is None else np.ascontiguousarray(q, np.float64)
        sigma = None if sigma is None else np.ascontiguousarray(sigma, np.float64)
        x = None if x is None else np.ascontiguousarray(x, np.float64)
        _check(lib().btam_batch_set_state(self.handle, int(k), _d(q), _d(sigma), _d(x)),
               "btam_batch_set_state")

    def autotune(self, precision=FP32C):
        v1, v2 = ctypes.c_int(), ctypes.c_int()
        _check(lib().btam_batch_autotune(self.handle, precision, ctypes.byref(v1),
                                         ctypes.byref(v2)), "btam_batch_autotune")
        return v1.value, v2.value

    def set_variants(self, precision, v1, v2):
        _check(lib().btam_batch_set_variants(self.handle, precision, int(v1), int(v2)),
               "btam_batch_set_variants")

    def evaluate_async(self, precision=FP32C):
        _check(lib().btam_batch_eval_async(self.handle, precision), "btam_batch_eval_async")

    def sync(self):
        _check(lib().btam_batch_sync(self.handle), "btam_batch_sync")

    def evaluate(self, precision=FP32C):
        """One evaluation of every system; returns the totals, shape (n_sys, 4)."""
        self.evaluate_async(precision)
        return self.totals()

    def totals(self):
        out = np.zeros((len(self.systems), 4))
        _check(lib().btam_batch_totals_copy(self.handle, _d(out)), "btam_batch_totals_copy")
        return out

    def results(self, k, want=("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals")):
        n = self.systems[k].n
        shapes = dict(rho=(n,), V0=(n,), S0=(n,), Rq=(n, 3), Rs=(n,), Rx=(n,), totals=(4,))
        out = {c: np.zeros(shapes[c]) for c in want}
        args = [_d(out.get(c)) for c in ("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals")]
        _check(lib().btam_batch_results_copy(self.handle, int(k), *args),
               "btam_batch_results_copy")
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().btam_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


JOB_RELAX, JOB_DMD, JOB_EVAL, JOB_STRETCH = 0, 1, 2, 3
RELAX_FP64, RELAX_MIXED, RELAX_FP32C, RELAX_NEWTON, RELAX_NGMRES = 0, 1, 2, 3, 4
MP_FD, MP_ANALYTIC = 1, 2


def estimate_bytes(sysdict):
    n = len(sysdict["x"])
    cell = np.ascontiguousarray(sysdict["cell"], np.float64).reshape(9)
    per = np.ascontiguousarray(sysdict["periodic"], np.int32)
    return int(lib().btam_estimate_bytes(n, _d(cell), _i(per)))


class Server:
    """Concurrent job server on the current device (btam_server_*)."""

    def __init__(self, tables, workers=8, budget_bytes=0):
        self.tables = tables
        h = _V()
        _check(lib().btam_server_create(tables.handle, int(workers), int(budget_bytes),
                                        ctypes.byref(h)), "btam_server_create")
        self.handle = h
        self.sizes = {}

    def submit(self, sysdict, kind, precision=FP32C, mode=RELAX_FP32C, tol=1e-5, max_iter=300,
               nsteps=100, dmd=(1e-3, 0.045, 3.2, 1e-8, 0.9), plain=False, history=0):
        """Queues a job; plain=True runs it on the plain two-pass kernel pair
        on its own instead of through the server's batched evaluations.
        history: the relaxation's L-BFGS history or N-GMRES subspace size
        (0: 8, or 3 for N-GMRES)."""
        s = sysdict
        arrs = dict(q=np.ascontiguousarray(s["q"], np.float64),
                    sigma=np.ascontiguousarray(s["sigma"], np.float64),
                    x=np.ascontiguousarray(s["x"], np.float64),
                    species=np.ascontiguousarray(s["species"], np.int32),
                    origin=np.ascontiguousarray(s["origin"], np.float64),
                    cell=np.ascontiguousarray(s["cell"], np.float64).reshape(9),
                    periodic=np.ascontiguousarray(s["periodic"], np.int32))
        for k in ("beta", "gamma"):
            if s.get(k) is not None:
                arrs[k] = np.ascontiguousarray(s[k], np.float64)
        sp = JobSpec()
        sp.kind, sp.precision, sp.mode, sp.n = int(kind), int(precision), int(mode), len(arrs["x"])
        for k in ("q", "sigma", "x", "origin", "cell", "beta", "gamma"):
            if k in arrs:
                setattr(sp, k, _d(arrs[k]))
        sp.species = _i(arrs["species"])
        sp.periodic = _i(arrs["periodic"])
        sp.tol, sp.max_iter, sp.nsteps = float(tol), int(max_iter), int(nsteps)
        sp.lbfgs_m = int(history)
        sp.plain = int(bool(plain))
        for c in range(5):
            sp.dmd_params[c] = float(dmd[c])
        jid = ctypes.c_longlong()
        _check(lib().btam_server_submit(self.handle, ctypes.byref(sp), ctypes.byref(jid)),
               "btam_server_submit")
        self.sizes[jid.value] = sp.n
        return jid.value

    def wait(self, job_id, timeout=-1.0):
        """Result dict of a job (its final state included); raises on a job
        error."""
        n = self.sizes.pop(job_id)
        res = JobResult()
        q = np.zeros((n, 3))
        sigma = np.zeros(n)
        x = np.zeros(n)
        _check(lib().btam_server_wait(self.handle, job_id, float(timeout), ctypes.byref(res),
                                      _d(q), _d(sigma), _d(x)), "btam_server_wait")
        out = {f: getattr(res, f) for f, _ in JobResult._fields_}
        out["h_quanta"] = (res.h_quanta_hi << 64) + (res.h_quanta_lo & 0xFFFFFFFFFFFFFFFF)
        out.update(q=q, sigma=sigma, x=x)
        return out

    def stats(self):
        w, c, f, b = (ctypes.c_longlong() for _ in range(4))
        r = ctypes.c_int()
        _check(lib().btam_server_stats(self.handle, ctypes.byref(w), ctypes.byref(r),
                                       ctypes.byref(c), ctypes.byref(f), ctypes.byref(b)),
               "btam_server_stats")
        return dict(waiting=w.value, running=r.value, completed=c.value, failed=f.value,
                    bytes_in_use=b.value)

    def batch_stats(self):
        """Continuous batching counters: rounds, job evaluations served,
        rebuilds of the shared batch."""
        r, e, b = (ctypes.c_longlong() for _ in range(3))
        _check(lib().btam_server_batch_stats(self.handle, ctypes.byref(r), ctypes.byref(e),
                                             ctypes.byref(b)), "btam_server_batch_stats")
        return dict(rounds=r.value, evaluations=e.value, rebuilds=b.value)

    def close(self):
        if getattr(self, "handle", None):
            lib().btam_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
