"""Shared test set-up: markers, import paths and library fixtures."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "bt-am_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

HOSTMODEL_DIR = os.path.join(ROOT, "tests", "hostmodel")
HOSTMODEL_SO = os.path.join(HOSTMODEL_DIR, "_build", "libbtam_hostmodel.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def build_hostmodel():
    src = os.path.join(HOSTMODEL_DIR, "hostmodel.cpp")
    deps = [src] + [os.path.join(ROOT, "bt-am_b200", "csrc", f)
                    for f in ("adp_core.cuh", "tables_io.hpp")]
    if (not os.path.exists(HOSTMODEL_SO) or
            any(os.path.getmtime(d) > os.path.getmtime(HOSTMODEL_SO) for d in deps)):
        os.makedirs(os.path.dirname(HOSTMODEL_SO), exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                        "-o", HOSTMODEL_SO, src], check=True)
    return HOSTMODEL_SO


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import pyoracle
    r = pyoracle.reference()
    if r is None:
        pytest.skip("reference build oracle/_ref absent (needs the reference tree)")
    return r


@pytest.fixture(scope="session")
def hostmodel():
    import hostmodel_py
    return hostmodel_py.HostModel(build_hostmodel())


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_tables():
    if not _gpu_available():
        pytest.skip("no CUDA device")
    import btam
    return btam.Tables()
