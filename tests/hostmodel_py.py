"""ctypes access to the host-compiled model of the kernel arithmetic
(tests/hostmodel/hostmodel.cpp).  Test infrastructure only."""
import ctypes
import os

import numpy as np

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
TABLES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "bt-am_b200", "data")


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


class HostModel:
    def __init__(self, path):
        self.lib = ctypes.CDLL(path)
        if self.lib.hm_load_tables(TABLES.encode()) != 0:
            raise RuntimeError("host model: cannot load tables")

    def evaluate(self, full, n_real, owner, offs, idx, fp32=False, sym=False):
        code = np.ascontiguousarray((full["species"] == 1).astype(np.int32))
        out = {k: np.zeros(n_real) for k in ("rho", "V0", "S0", "selfx", "Rs", "Rx")}
        Rq = np.zeros((n_real, 3))
        self.lib.hm_eval(int(fp32), int(sym), len(full["x"]), n_real, _d(full["q"]), _d(full["sigma"]),
                         _d(full["x"]), _i(code), _d(full["beta"]), _d(full["gamma"]),
                         _i(owner), _i(offs), _i(idx), _d(out["rho"]), _d(out["V0"]),
                         _d(out["S0"]), _d(out["selfx"]), _d(Rq), _d(out["Rs"]),
                         _d(out["Rx"]))
        out["Rq"] = Rq
        return out
