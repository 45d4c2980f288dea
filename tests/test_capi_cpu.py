"""The C-ABI library without a GPU: it loads and exports every entry point
include/btam.h declares; the dump reader/writer round-trips; synthetic
workloads have the advertised sizes."""
import ctypes
import os

import numpy as np

import btam
from btam import dump, lattice


def test_library_exports_every_declared_symbol():
    names = btam.exported_symbols()
    assert len(names) >= 20
    # RTLD_NOW: every symbol the library needs resolves at load, not at the
    # first call
    L = ctypes.CDLL(btam.LIB_PATH, mode=os.RTLD_NOW | os.RTLD_LOCAL)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.btam_version() >= 100
    L.btam_status_string.restype = ctypes.c_char_p
    assert L.btam_status_string(3) == b"more than maxneigh neighbours"
    # no CUDA error has been turned into a status on this thread
    L.btam_last_cuda_error.restype = ctypes.c_char_p
    assert L.btam_last_cuda_error() == b""


def test_bindings_cover_header():
    assert set(btam.exported_symbols()) <= set(btam._PROTOS)


def test_dump_round_trip(tmp_path):
    s = lattice.supercell(4, 3, 3, ortho=True, h_fraction=0.3, x_range=(0.0, 0.4), seed=2)
    p = tmp_path / "s.dump"
    dump.write_dump(str(p), s)
    t = dump.read_dump(str(p))
    for k in ("q", "sigma", "x", "species", "beta", "gamma", "origin", "cell", "periodic"):
        assert np.array_equal(np.asarray(s[k]), np.asarray(t[k])), k


def test_workload_sizes():
    c1 = lattice.config1()
    assert (c1["species"] == 12).sum() == 250
    assert 80 <= (c1["species"] == 1).sum() <= 120
    c2 = lattice.supercell(20, 15, 15, with_tetra=True)
    assert (c2["species"] == 12).sum() == 9000 and (c2["species"] == 1).sum() == 18000


def test_plugin_table_adapter_builds():
    """include/btam_dmd_equations.hpp compiles against the reference's type
    declarations (the oracle's shim of Macros.hpp and of Eigen) into a
    reference-style caller, and that caller links against libbtam.so."""
    import compat_build
    assert os.path.exists(compat_build.build_probe())
